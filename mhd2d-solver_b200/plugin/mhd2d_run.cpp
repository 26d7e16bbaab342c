// mhd2d_run: the reference solver's program around the drop-in classes.
//
//   mhd2d_run [--backend=cpu|cuda] [--divb=host|device] config.ini
//
// Reads the same INI deck with the reference's own inputData
// (file_access.cpp:61-270, compiled unmodified), builds the problem with the
// reference's problem setups, and writes the same grid / non-grid /
// characteristics files with the reference's own writers
// (file_access.cpp:1091-1736, conversions.cpp).  The main loop follows
// main.cpp:66-360: output cadence by step or time, the div B cleaning loop,
// the NaN stop and the end-of-run report.
//
// --backend=cpu   SpatialMethodEnoRoe / EnoLF / CentralFD2 and
//                 TimeIntegrationRK3 / Euler (the reference's own classes);
// --backend=cuda  CudaSpatialMethod* and CudaTimeIntegration* from
//                 cuda_methods.hpp (the default).
// --divb=host     divBCalculation / divBCorrectionSOR of div_b_fix.cpp on
//                 the host state (the reference's lexicographic SOR);
// --divb=device   the same cleaning loop on the GPU through the C ABI
//                 (mhd_divb_calc / mhd_divb_sor: red-black SOR, the same
//                 stop rules), cuda backend only (the default there).
// With --divb=host both backends write byte-identical files.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>

#include "mhd2d.hpp"
#include "spatialmethodcentralfd2.hpp"
#include "spatialmethodenolf.hpp"
#include "spatialmethodenoroe.hpp"
#include "timeintegrationeuler.hpp"
#include "timeintegrationrk3.hpp"

#include "cuda_methods.hpp"
#include "mhd2d_b200.h"

// The reference's reader and writers report fatal input errors through this
// function, which its program defines (main.cpp:365-396): print the message
// and exit with the code of the status class.
void criticalError(ReturnStatus error, const std::string message) {
  ERROUT << "Critical error!\n"
         << ">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>\n"
         << message << "\n"
         << ">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>\n"
         << "Terminating execution.\n";
  int code = 0;
  switch (error) {
    case ReturnStatus::ErrorNotImplemented: code = 100; break;
    case ReturnStatus::ErrorTimeUnderflow: code = 101; break;
    case ReturnStatus::ErrorNotConverged: code = 102; break;
    case ReturnStatus::ErrorNegativeDensity: code = 103; break;
    case ReturnStatus::ErrorNegativePressure: code = 104; break;
    case ReturnStatus::ErrorFileNotFound: code = 200; break;
    case ReturnStatus::ErrorFailedToParse: code = 201; break;
    case ReturnStatus::ErrorWrongParameter: code = 202; break;
    default: code = 0; break;
  }
  std::exit(code);
}

namespace {

struct Options {
  bool cuda = true;
  bool divb_device = true;
  const char* ini = nullptr;
};

Options parse_args(int argc, char** argv) {
  Options o;
  bool divb_given = false;
  for (int a = 1; a < argc; a++) {
    const std::string s = argv[a];
    if (s == "--backend=cpu") o.cuda = false;
    else if (s == "--backend=cuda") o.cuda = true;
    else if (s == "--divb=host") { o.divb_device = false; divb_given = true; }
    else if (s == "--divb=device") { o.divb_device = true; divb_given = true; }
    else if (s.size() > 2 && s[0] == '-' && s[1] == '-') {
      ERROUT << "unknown option " << s << LF;
      std::exit(2);
    } else {
      o.ini = argv[a];
    }
  }
  if (!o.cuda) {
    if (divb_given && o.divb_device) {
      ERROUT << "--divb=device needs --backend=cuda" << LF;
      std::exit(2);
    }
    o.divb_device = false;
  }
  return o;
}

// div B cleaning of one step (main.cpp:207-242), on the host state with the
// reference's functions or on the device through the stepper's context.
class DivBCleaner {
 public:
  DivBCleaner(const t_params& params, mhd_ctx* ctx) : params_(params), ctx_(ctx) {}

  void clean(t_data& data, int step) {
    if (params_.divb_method != DivBCorrectionMethod::SOR || params_.divb_sor_steps <= 0) return;
    if (ctx_ && mhd_upload(ctx_, data.U[0][0]) != MHD_OK) fail("mhd_upload");
    double divbsum = 0.0, divbmax = 0.0;
    for (int i = 0; i < params_.divb_sor_steps; i++) {
      calc(data, divbmax, divbsum);
      if (params_.log_params.divb_step)
        OUT << "divb corrector, step #" << step << ", loop #" << i << ": divbmax = " << divbmax
            << "\n";
      if (divbmax < params_.divb_sor_max) {
        if (params_.log_params.divb_step)
          OUT << "divb corrector, step #" << step << ": divb converged in " << i << " steps.\n";
        break;
      }
      if (sor(data) == ReturnStatus::ErrorNotConverged) {
        ERROUT << "WARNING: Div B corrector, r failed to converge.\n";
        break;
      }
    }
    calc(data, divbmax, divbsum);
    if (ctx_ && mhd_download(ctx_, data.U[0][0]) != MHD_OK) fail("mhd_download");
    if (divbmax > params_.divb_sor_max)
      ERROUT << "WARNING: Div B corrector failed to converge: divbmax = " << divbmax << "\n"
             << "         Simulation resumed, but B may be erroneous." << LF;
  }

 private:
  void calc(t_data& data, double& mx, double& sum) {
    if (!ctx_) {
      divBCalculation(data.U, params_, mx, sum);
      return;
    }
    if (mhd_divb_calc(ctx_, &mx, &sum) != MHD_OK) fail("mhd_divb_calc");
  }

  ReturnStatus sor(t_data& data) {
    if (!ctx_) return divBCorrectionSOR(data.U, params_).status;
    mhd_sor_params p{};
    p.divb_skip_steps = params_.divb_skip_steps;
    p.sor_steps = params_.divb_sor_steps;
    p.sor_rsteps = params_.divb_sor_rsteps;
    p.sor_rmax = params_.divb_sor_rmax;
    p.sor_divbmax = params_.divb_sor_max;
    p.omega_use_static = params_.divb_sor_omega_use_static ? 1 : 0;
    p.omega = params_.divb_sor_omega;
    int sweeps = 0;
    const int st = mhd_divb_sor(ctx_, &p, &sweeps);
    if (st == MHD_ERR_NOT_CONVERGED) return ReturnStatus::ErrorNotConverged;
    if (st != MHD_OK) fail("mhd_divb_sor");
    if (params_.log_params.r_end) OUT << "SOR: converged in " << sweeps << " sweeps\n";
    return ReturnStatus::OK;
  }

  void fail(const char* what) {
    char msg[512] = {0};
    int is_error = 0;
    mhd_last_error(ctx_, msg, sizeof msg, &is_error);
    criticalError(ReturnStatus::ErrorNotImplemented,
                  std::string("div B cleaning on the device: ") + what + ": " + msg);
  }

  const t_params& params_;
  mhd_ctx* ctx_;
};

std::unique_ptr<SpatialIntegrationMethod> make_method(const Options& o, const t_params& params,
                                                      size_t halo, t_boundary b) {
  using Ptr = std::unique_ptr<SpatialIntegrationMethod>;
  const size_t nx = params.nx, ny = params.ny;
  switch (params.scheme) {
    case IntegrationMethod::CentralFD:
      return o.cuda ? Ptr(new CudaSpatialMethodCentralFD2(nx, ny, halo, params.dx, params.dy, b,
                                                           params.gamma))
                    : Ptr(new SpatialMethodCentralFD2(nx, ny, halo, params.dx, params.dy, b,
                                                      params.gamma));
    case IntegrationMethod::ENO_Roe:
      return o.cuda ? Ptr(new CudaSpatialMethodEnoRoe(nx, ny, halo, params.dx, params.dy, b,
                                                      params.gamma))
                    : Ptr(new SpatialMethodEnoRoe(nx, ny, halo, params.dx, params.dy, b,
                                                  params.gamma));
    case IntegrationMethod::ENO_LF:
      return o.cuda ? Ptr(new CudaSpatialMethodEnoLF(nx, ny, halo, params.dx, params.dy, b,
                                                     params.gamma))
                    : Ptr(new SpatialMethodEnoLF(nx, ny, halo, params.dx, params.dy, b,
                                                 params.gamma));
    default:
      criticalError(ReturnStatus::ErrorWrongParameter,
                    std::string{} + "main: Unknown space integration method.");
  }
  return Ptr();
}

std::unique_ptr<TimeIntegrationMethod> make_stepper(const Options& o, const t_params& params,
                                                    size_t halo,
                                                    std::unique_ptr<SpatialIntegrationMethod> m) {
  using Ptr = std::unique_ptr<TimeIntegrationMethod>;
  const size_t nx = params.nx, ny = params.ny;
  const double lo = params.dt_min, hi = params.dt_max, cfl = params.cfl_number;
  switch (params.time_stepping) {
    case TimeStepMethod::Euler:
      return o.cuda ? Ptr(new CudaTimeIntegrationEuler(nx, ny, halo, lo, hi, cfl, std::move(m)))
                    : Ptr(new TimeIntegrationEuler(nx, ny, halo, lo, hi, cfl, std::move(m)));
    case TimeStepMethod::RungeKutta3_TVD:
      return o.cuda ? Ptr(new CudaTimeIntegrationRK3(nx, ny, halo, lo, hi, cfl, std::move(m)))
                    : Ptr(new TimeIntegrationRK3(nx, ny, halo, lo, hi, cfl, std::move(m)));
    default:
      criticalError(ReturnStatus::ErrorWrongParameter,
                    std::string{} + "main: Unknown time stepping method.");
  }
  return Ptr();
}

// Whether this step writes a file: by step count, or once the simulated
// time passes the next mark (which then moves past it).
bool due(WriteSkipMode mode, int step, int skip_steps, double t, double skip_t, double& mark,
         const char* what) {
  switch (mode) {
    case WriteSkipMode::Step:
      return step % skip_steps == 0;
    case WriteSkipMode::Time: {
      const bool hit = t >= mark;
      while (hit && mark <= t) mark += skip_t;
      return hit;
    }
    default:
      criticalError(ReturnStatus::ErrorWrongParameter,
                    std::string{} + "main: Unknown " + what + " output mode.");
  }
  return false;
}

}  // namespace

int main(int argc, char** argv) {
  namespace chr = std::chrono;
  const Options opt = parse_args(argc, argv);
  if (!opt.ini) {
    OUT << "Usage: " << argv[0] << " [--backend=cpu|cuda] [--divb=host|device] config_file\n";
    return 0;
  }
  const auto t_start = chr::steady_clock::now();

  t_output out_grid, out_nongrid, out_chars;
  t_params params;
  t_data data;
  inputData(opt.ini, out_grid, out_nongrid, params, data);
  out_chars = out_grid;
  out_chars.single_file = false;
  out_chars.binary = true;
  out_chars.filename = std::string{"char-"} + out_grid.filename;
  if (out_grid.single_file) openFile(out_grid);
  openFile(out_nongrid);
  outputGridData(out_grid, params, data, 0, 0);
  outputNonGridData(out_nongrid, params, data, 0, 0);

  const size_t halo = size_t{NXFIRST};
  const t_boundary boundary{params.boundary[params.b_right], params.boundary[params.b_top],
                            params.boundary[params.b_left], params.boundary[params.b_bottom]};
  auto method = make_method(opt, params, halo, boundary);
  method->initializeDirichletBoundaries(data.U);
  mhd_ctx* ctx = nullptr;
  if (opt.cuda) ctx = static_cast<CudaSpatialMethod*>(method.get())->context();
  auto stepper = make_stepper(opt, params, halo, std::move(method));
  DivBCleaner cleaner(params, opt.divb_device ? ctx : nullptr);

  const int progress_every =
      params.time_mode == TimeStepMode::Constant ? (params.steps > 100 ? params.steps / 100 : 1) : 0;
  double mark_grid = out_grid.skip_t, mark_nongrid = out_nongrid.skip_t;
  double mark_screen = params.t_max / 100.0;
  int step = 1, record = 1;
  bool done = false;

  const auto t_loop = chr::steady_clock::now();
  OUT << "@ t = " << chr::duration<double>(t_loop - t_start).count() << " sec : Init finished.\n";
  while (!done) {
    const t_status st =
        stepper->step(data.U, data.cx, data.cy, data.LUx, data.LUy, data.borderFlux, data.dt);
    if (st.status == ReturnStatus::ErrorTimeUnderflow) {
      ERROUT << "ERROR: main: Time step size smaller than the smallest allowed value.\n"
             << "       Reached at step #" << step << ", at t = " << data.t_current << ".\n"
             << "       The simulation will now terminate." << LF;
      break;
    }
    if (st.isError) {
      ERROUT << "ERROR: main: Terminating simulation." << LF;
      ERROUT << st.message;
      break;
    }
    if (step % params.divb_skip_steps == 0) cleaner.clean(data, step);
    data.t_current += data.dt;

    bool to_screen = false;
    switch (params.time_mode) {
      case TimeStepMode::Constant:
        done = step == params.steps;
        to_screen = step % progress_every == 0;
        break;
      case TimeStepMode::Variable:
        done = data.t_current >= params.t_max;
        to_screen = data.t_current >= mark_screen;
        while (to_screen && mark_screen <= data.t_current) mark_screen += params.t_max / 100.0;
        break;
      default:
        criticalError(ReturnStatus::ErrorWrongParameter,
                      std::string{} + "main: Unknown time stepping mode.");
    }
    const bool to_file = due(out_grid.skip_mode, step, out_grid.skip_steps, data.t_current,
                             out_grid.skip_t, mark_grid, "grid");
    const bool to_nongrid = due(out_nongrid.skip_mode, step, out_nongrid.skip_steps,
                                data.t_current, out_nongrid.skip_t, mark_nongrid, "non-grid");
    if (to_file || to_nongrid) toNaturalData(params, data);
    if (to_file) {
      outputGridData(out_grid, params, data, step, record++);
      if (params.log_params.characteristics && step > 0 &&
          (params.scheme == IntegrationMethod::ENO_Roe ||
           params.scheme == IntegrationMethod::ENO_LF))
        outputCharacteristicsBinary(out_chars, params, data.cx, data.cy, data.LUx, data.LUy,
                                    data.t_current, step, record);
    }
    if (to_nongrid) outputNonGridData(out_nongrid, params, data, step, record);

    if (to_screen) {
      const double el = chr::duration<double>(chr::steady_clock::now() - t_start).count();
      if (params.time_mode == TimeStepMode::Constant)
        OUT << "@ t = " << el << " sec : " << step << " / " << params.steps << " steps ("
            << (100.0 * step / params.steps) << "%) done." << LF;
      else
        OUT << "@ t = " << el << " sec : " << step << " steps done, " << data.t_current << " / "
            << params.t_max << " simulated time (" << (100.0 * data.t_current / params.t_max)
            << "%)." << LF;
    }
    if (std::isnan(data.U[0][NXFIRST][NYFIRST])) {
      ERROUT << "WARNING: NaN detected. Stopping simulation at step " << step
             << ", t = " << data.t_current << ", with " << record - 1 << " grids recorded."
             << LF;
      done = true;
    }
    step++;
  }

  if (out_grid.single_file) closeFile(out_grid);
  closeFile(out_nongrid);
  const double total = chr::duration<double>(chr::steady_clock::now() - t_start).count();
  const double loop = chr::duration<double>(chr::steady_clock::now() - t_loop).count();
  OUT << "@ t = " << total << " sec : Simulation finished.\n"
      << " - Backend            : " << (opt.cuda ? "cuda" : "cpu")
      << (opt.divb_device ? " (div B on the device)" : "") << "\n"
      << " - Grids recorded     : " << record - 1 << "\n"
      << " - Successful steps   : " << step - 1 << "\n"
      << " - Simulated time     : " << data.t_current << "\n"
      << " - Main loop duration : " << loop << " seconds\n"
      << " - Time step average  : " << loop / (step - 1) << " seconds.\n";
  return 0;
}
