// Drop-in subclasses of the reference solver's plugin interfaces that run
// the time-step hot path on a B200 through libmhd2d_b200.so.
//
//   CudaSpatialMethodEnoRoe / CudaSpatialMethodEnoLF / CudaSpatialMethodCentralFD2
//       : SpatialIntegrationMethod
//       (spatialintegrationmethod.hpp:6-65) — integrate() uploads U, runs the
//       boundary fill and the fused flux kernel, downloads U (ghosts filled)
//       and UL, like SpatialMethodEnoRoe/EnoLF::integrate.
//   CudaTimeIntegrationRK3 / CudaTimeIntegrationEuler : TimeIntegrationMethod
//       (timeintegrationmethod.hpp:6-53) — step() runs the whole RK3 / Euler
//       step (three spatial operators, CFL control with the power-of-two dt
//       and retry semantics, stage updates) on the device: one upload and one
//       download of U per step.  The method passed in must be one of the
//       Cuda spatial methods; the stepper takes over its device context.
//
// Built against the reference's own headers (mhd2d.hpp and the interface
// headers).  A caller selects these classes where main.cpp:124-151 builds
// its method and stepper.  Errors come back as the reference's t_status;
// a CUDA failure carries kCudaFailure, a status value outside the
// reference's enumerators, with isError set and the CUDA error text.
#ifndef MHD2D_B200_CUDA_METHODS_HPP
#define MHD2D_B200_CUDA_METHODS_HPP

#include <memory>

#include "spatialintegrationmethod.hpp"
#include "timeintegrationmethod.hpp"

struct mhd_ctx;

// Status of a failed CUDA call (an allocation, a launch, a copy).  The
// reference's ReturnStatus has no such member and none of its members means
// it, so the value is one past them; it compares unequal to every
// reference status, and main.cpp's loop treats it as any other isError.
constexpr ReturnStatus kCudaFailure = static_cast<ReturnStatus>(100);

class CudaSpatialMethod : public SpatialIntegrationMethod {
 public:
  CudaSpatialMethod(size_t nx, size_t ny, size_t bufferWidth, double dx, double dy,
                    t_boundary boundary, double gamma, int scheme, bool characteristics = true);
  ~CudaSpatialMethod() override;

  t_status integrate(t_matrices U, t_matrices UL, borderVectors borderFlux,
                     double& dtIdeal) override;
  bool getCharacteristicsX(t_matrices cx, t_matrices LUx) override;
  bool getCharacteristicsY(t_matrices cy, t_matrices LUy) override;

  mhd_ctx* context() { return ctx_; }
  // Hands the Dirichlet snapshot taken by initializeDirichletBoundaries to
  // the device (no-op when no side is Dirichlet or it was already sent).
  t_status syncBoundaries();

 protected:
  mhd_ctx* ctx_ = nullptr;
  bool characteristics_;
  bool dirichletSent_ = false;
};

class CudaSpatialMethodEnoRoe : public CudaSpatialMethod {
 public:
  CudaSpatialMethodEnoRoe(size_t nx, size_t ny, size_t bufferWidth, double dx, double dy,
                          t_boundary boundary, double gamma)
      : CudaSpatialMethod(nx, ny, bufferWidth, dx, dy, boundary, gamma, 2) {}
};

class CudaSpatialMethodEnoLF : public CudaSpatialMethod {
 public:
  CudaSpatialMethodEnoLF(size_t nx, size_t ny, size_t bufferWidth, double dx, double dy,
                         t_boundary boundary, double gamma)
      : CudaSpatialMethod(nx, ny, bufferWidth, dx, dy, boundary, gamma, 3) {}
};

// SpatialMethodCentralFD2 (spatialmethodcentralfd2.cpp): second-order
// central differences; it keeps no characteristics.
class CudaSpatialMethodCentralFD2 : public CudaSpatialMethod {
 public:
  CudaSpatialMethodCentralFD2(size_t nx, size_t ny, size_t bufferWidth, double dx, double dy,
                              t_boundary boundary, double gamma)
      : CudaSpatialMethod(nx, ny, bufferWidth, dx, dy, boundary, gamma, 1, false) {}
};

class CudaTimeIntegration : public TimeIntegrationMethod {
 public:
  CudaTimeIntegration(size_t nx, size_t ny, size_t bufferWidth, double dtMin, double dtMax,
                      double cflNumber, std::unique_ptr<SpatialIntegrationMethod> method,
                      int timeMethod);
  t_status step(t_matrices U, t_matrices cx, t_matrices cy, t_matrices LUx, t_matrices LUy,
                borderVectors borderFlux, double& dtCurrent) override;

 protected:
  CudaSpatialMethod* cuda_ = nullptr;
};

class CudaTimeIntegrationRK3 : public CudaTimeIntegration {
 public:
  CudaTimeIntegrationRK3(size_t nx, size_t ny, size_t bufferWidth, double dtMin, double dtMax,
                         double cflNumber, std::unique_ptr<SpatialIntegrationMethod> method)
      : CudaTimeIntegration(nx, ny, bufferWidth, dtMin, dtMax, cflNumber, std::move(method), 2) {}
};

class CudaTimeIntegrationEuler : public CudaTimeIntegration {
 public:
  CudaTimeIntegrationEuler(size_t nx, size_t ny, size_t bufferWidth, double dtMin, double dtMax,
                           double cflNumber, std::unique_ptr<SpatialIntegrationMethod> method)
      : CudaTimeIntegration(nx, ny, bufferWidth, dtMin, dtMax, cflNumber, std::move(method), 1) {}
};

#endif
