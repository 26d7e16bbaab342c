// Drop-in subclasses of the reference plugin interfaces (see cuda_methods.hpp).
#include "cuda_methods.hpp"

#include <stdexcept>
#include <string>

#include "mhd2d_b200.h"

namespace {

t_status status_from(mhd_ctx* ctx, int st, const char* where) {
  char msg[1024] = {0};
  int is_error = 0;
  mhd_last_error(ctx, msg, sizeof msg, &is_error);
  t_status s{is_error != 0, st == MHD_ERR_CUDA ? kCudaFailure : static_cast<ReturnStatus>(st),
             std::string(msg)};
  if (st == MHD_ERR_CUDA) s.isError = true;
  if (st != MHD_OK) s.message += std::string("\n! ") + where;
  return s;
}

}  // namespace

CudaSpatialMethod::CudaSpatialMethod(size_t nx, size_t ny, size_t bufferWidth, double dx, double dy,
                                     t_boundary boundary, double gamma, int scheme,
                                     bool characteristics)
    : SpatialIntegrationMethod{nx, ny, bufferWidth, dx, dy, boundary, gamma},
      characteristics_(characteristics) {
  if (bufferWidth < (scheme == 1 ? 1u : 2u))
    throw std::domain_error(scheme == 1 ? "Buffer is too small for second order central finite "
                                          "difference; need at least 1 extra grid"
                                        : "Buffer is too small for ENO; need at least 2 extra grids");
  if (bufferWidth != 2)
    throw std::domain_error("the device layout has exactly 2 ghost cells per side");
  const int bc[4] = {int(boundary.left), int(boundary.right), int(boundary.bottom),
                     int(boundary.top)};
  const int st = mhd_ctx_create(int(nx), int(ny), 2, dx, dy, gamma, bc, scheme, 2, 0.0, 1.0, 0.0,
                                characteristics ? MHD_FLAG_CHARACTERISTICS : 0, 0, &ctx_);
  if (st != MHD_OK)
    throw std::runtime_error("mhd_ctx_create failed with status " + std::to_string(st));
}

CudaSpatialMethod::~CudaSpatialMethod() { mhd_ctx_destroy(ctx_); }

t_status CudaSpatialMethod::syncBoundaries() {
  if (requireBoundaryInitialization)  // spatialintegrationmethod.cpp:88-90
    return {true, ReturnStatus::ErrorWrongParameter,
            "SpatialIntegrationMethod::applyBoundaryConditions: boundary not initialized."};
  const bool dirichlet = boundary.left == BoundaryCondition::Dirichlet ||
                         boundary.right == BoundaryCondition::Dirichlet ||
                         boundary.bottom == BoundaryCondition::Dirichlet ||
                         boundary.top == BoundaryCondition::Dirichlet;
  if (dirichlet && !dirichletSent_) {
    const int st = mhd_set_dirichlet(ctx_, dirichletBoundaryLeft[0], dirichletBoundaryRight[0],
                                     dirichletBoundaryBottom[0], dirichletBoundaryTop[0]);
    if (st != MHD_OK) return status_from(ctx_, st, "CudaSpatialMethod::syncBoundaries");
    dirichletSent_ = true;
  }
  return {false, ReturnStatus::OK, ""};
}

t_status CudaSpatialMethod::integrate(t_matrices U, t_matrices UL, borderVectors /*borderFlux*/,
                                      double& dtIdeal) {
  t_status s = syncBoundaries();
  if (s.isError) {
    s.message += "\n! CudaSpatialMethod::integrate";
    return s;
  }
  const int st = mhd_integrate_host(ctx_, U[0][0], UL[0][0], &dtIdeal);
  return status_from(ctx_, st, "CudaSpatialMethod::integrate");
}

bool CudaSpatialMethod::getCharacteristicsX(t_matrices cx, t_matrices LUx) {
  if (!characteristics_) return false;
  return mhd_get_characteristics(ctx_, cx[0][0], nullptr, LUx[0][0], nullptr) == MHD_OK;
}

bool CudaSpatialMethod::getCharacteristicsY(t_matrices cy, t_matrices LUy) {
  if (!characteristics_) return false;
  return mhd_get_characteristics(ctx_, nullptr, cy[0][0], nullptr, LUy[0][0]) == MHD_OK;
}

CudaTimeIntegration::CudaTimeIntegration(size_t nx, size_t ny, size_t bufferWidth, double dtMin,
                                         double dtMax, double cflNumber,
                                         std::unique_ptr<SpatialIntegrationMethod> m,
                                         int timeMethod)
    : TimeIntegrationMethod{nx, ny, bufferWidth, dtMin, dtMax, cflNumber, std::move(m)} {
  cuda_ = dynamic_cast<CudaSpatialMethod*>(method.get());
  if (!cuda_)
    throw std::invalid_argument("CudaTimeIntegration needs a CudaSpatialMethod to drive");
  if (mhd_set_stepper(cuda_->context(), timeMethod, dtMin, dtMax, cflNumber) != MHD_OK)
    throw std::runtime_error("mhd_set_stepper failed");
}

t_status CudaTimeIntegration::step(t_matrices U, t_matrices cx, t_matrices cy, t_matrices LUx,
                                   t_matrices LUy, borderVectors /*borderFlux*/,
                                   double& dtCurrent) {
  t_status s = cuda_->syncBoundaries();
  if (s.isError) {
    s.message += "\n! CudaTimeIntegration::step";
    return s;
  }
  double dt = dtCurrent;
  const int st = mhd_step_host(cuda_->context(), U[0][0], &dt);
  if (st != MHD_OK) return status_from(cuda_->context(), st, "CudaTimeIntegration::step");
  dtCurrent = dt;
  method->getCharacteristicsX(cx, LUx);  // timeintegrationrk3.cpp:151-152
  method->getCharacteristicsY(cy, LUy);
  return {false, ReturnStatus::OK, ""};
}
