// Drop-in check: the same run three ways, compared bit for bit.
//   A  reference TimeIntegrationRK3 + reference SpatialMethodEnoRoe/EnoLF/CentralFD2
//   B  reference TimeIntegrationRK3 + CudaSpatialMethodEnoRoe/EnoLF/CentralFD2
//   C  CudaTimeIntegrationRK3      + CudaSpatialMethodEnoRoe/EnoLF/CentralFD2
// usage: plugin_check <scheme 1|2|3> <problem ot|bw|dir> <steps>
// Prints one line per comparison and exits non-zero on any difference.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "cuda_methods.hpp"
#include "spatialmethodcentralfd2.hpp"
#include "spatialmethodenolf.hpp"
#include "spatialmethodenoroe.hpp"
#include "timeintegrationrk3.hpp"

namespace {

struct Block {
  int n, sx, sy;
  std::vector<double> data;
  std::vector<double*> rows;
  std::vector<double**> planes;
  Block(int n_, int sx_, int sy_) : n(n_), sx(sx_), sy(sy_), data(size_t(n_) * sx_ * sy_, 0.0),
                                     rows(size_t(n_) * sx_), planes(n_) {
    for (int k = 0; k < n; k++) {
      planes[k] = &rows[size_t(k) * sx];
      for (int i = 0; i < sx; i++) rows[size_t(k) * sx + i] = data.data() + (size_t(k) * sx + i) * sy;
    }
  }
  t_matrices m() { return planes.data(); }
};

struct Vecs {
  std::vector<double> data;
  std::vector<double*> rows;
  Vecs(int n, int s) : data(size_t(n) * s, 0.0), rows(n) {
    for (int k = 0; k < n; k++) rows[k] = data.data() + size_t(k) * s;
  }
  t_vectors v() { return rows.data(); }
};

struct Problem {
  int nx, ny;
  double dx, dy, gamma, dt0, dtmax, cfl;
  t_boundary b;
  std::vector<double> U;
};

void conserved(Problem& p, int i, int j, double r, double u, double v, double w, double bx,
               double by, double bz, double pr) {
  const int NXT = p.nx + 4, NYT = p.ny + 4;
  auto at = [&](int k) -> double& { return p.U[(size_t(k) * NXT + i) * NYT + j]; };
  at(0) = r; at(1) = u * r; at(2) = v * r; at(3) = w * r;
  at(4) = bx; at(5) = by; at(6) = bz;
  at(7) = pr / (p.gamma - 1.0) + 0.5 * r * (u * u + v * v + w * w) + 0.5 * (bx * bx + by * by + bz * bz);
}

Problem make(const std::string& name) {
  Problem p{};
  if (name == "ot") {
    p.nx = p.ny = 64; p.gamma = 5.0 / 3.0; p.dx = p.dy = 2 * M_PI / 64;
    p.dt0 = p.dtmax = 0.03125; p.cfl = 0.4;
    p.b = t_boundary{BoundaryCondition::Periodic, BoundaryCondition::Periodic,
                     BoundaryCondition::Periodic, BoundaryCondition::Periodic};
  } else if (name == "bw") {
    p.nx = 128; p.ny = 8; p.gamma = 2.0; p.dx = 2.0 / 128; p.dy = 0.5 / 8;
    p.dt0 = p.dtmax = 0.0078125; p.cfl = 0.4;
    p.b = t_boundary{BoundaryCondition::Neumann, BoundaryCondition::Neumann,
                     BoundaryCondition::Neumann, BoundaryCondition::Neumann};
  } else {  // a blast with Dirichlet / open / Neumann / periodic sides
    p.nx = 48; p.ny = 40; p.gamma = 5.0 / 3.0; p.dx = 1.0 / 48; p.dy = 1.0 / 40;
    p.dt0 = p.dtmax = 0.01; p.cfl = 0.4;
    // t_boundary order: right, top, left, bottom
    p.b = t_boundary{BoundaryCondition::Open, BoundaryCondition::Dirichlet,
                     BoundaryCondition::Dirichlet, BoundaryCondition::Neumann};
  }
  p.U.assign(size_t(8) * (p.nx + 4) * (p.ny + 4), 0.0);
  for (int i = 2; i < p.nx + 2; i++)
    for (int j = 2; j < p.ny + 2; j++) {
      const double x = (i - 2) * p.dx, y = (j - 2) * p.dy;
      if (name == "ot") {
        conserved(p, i, j, p.gamma * p.gamma, -std::sin(y), std::sin(x), 0.0, -std::sin(y),
                  std::sin(2 * x), 0.0, p.gamma);
      } else if (name == "bw") {
        const bool left = (i - 2) * p.dx < 1.0 - 0.5 * p.dx;
        conserved(p, i, j, left ? 1.0 : 0.125, 0, 0, 0, 0.75, left ? 1.0 : -1.0, 0.0, left ? 1.0 : 0.1);
      } else {
        const double rx = x - 0.5, ry = y - 0.5, in = (rx * rx + ry * ry < 0.01) ? 1.0 : 0.0;
        conserved(p, i, j, in ? 1.0 : 0.125, 0.1, -0.05, 0.02, 0.7, 0.7, 0.1, in ? 10.0 : 1.0);
      }
    }
  return p;
}

enum Mode { REF, REF_STEPPER_CUDA_METHOD, CUDA };

std::vector<double> run(const Problem& p, int scheme, Mode mode, int steps, double* dt_out,
                        std::vector<double>* chars) {
  const int NXT = p.nx + 4, NYT = p.ny + 4;
  Block U(8, NXT, NYT), cx(8, NXT, NYT), cy(8, NXT, NYT), lx(8, NXT, NYT), ly(8, NXT, NYT);
  std::memcpy(U.data.data(), p.U.data(), p.U.size() * sizeof(double));
  std::unique_ptr<SpatialIntegrationMethod> m;
  if (mode == REF) {
    if (scheme == 3) m.reset(new SpatialMethodEnoLF(p.nx, p.ny, 2, p.dx, p.dy, p.b, p.gamma));
    else if (scheme == 1) m.reset(new SpatialMethodCentralFD2(p.nx, p.ny, 2, p.dx, p.dy, p.b, p.gamma));
    else m.reset(new SpatialMethodEnoRoe(p.nx, p.ny, 2, p.dx, p.dy, p.b, p.gamma));
  } else {
    if (scheme == 3) m.reset(new CudaSpatialMethodEnoLF(p.nx, p.ny, 2, p.dx, p.dy, p.b, p.gamma));
    else if (scheme == 1)
      m.reset(new CudaSpatialMethodCentralFD2(p.nx, p.ny, 2, p.dx, p.dy, p.b, p.gamma));
    else m.reset(new CudaSpatialMethodEnoRoe(p.nx, p.ny, 2, p.dx, p.dy, p.b, p.gamma));
  }
  m->initializeDirichletBoundaries(U.m());
  std::unique_ptr<TimeIntegrationMethod> s;
  if (mode == CUDA)
    s.reset(new CudaTimeIntegrationRK3(p.nx, p.ny, 2, 1e-9, p.dtmax, p.cfl, std::move(m)));
  else
    s.reset(new TimeIntegrationRK3(p.nx, p.ny, 2, 1e-9, p.dtmax, p.cfl, std::move(m)));
  Vecs bl(8, NYT), br(8, NYT), bu(8, NXT), bd(8, NXT);
  borderVectors bf{bl.v(), br.v(), bu.v(), bd.v()};
  double dt = p.dt0;
  for (int n = 0; n < steps; n++) {
    t_status st = s->step(U.m(), cx.m(), cy.m(), lx.m(), ly.m(), bf, dt);
    if (st.isError) {
      std::fprintf(stderr, "step %d failed: %s\n", n, st.message.c_str());
      std::exit(3);
    }
  }
  *dt_out = dt;
  chars->clear();
  for (Block* b : {&cx, &cy, &lx, &ly}) chars->insert(chars->end(), b->data.begin(), b->data.end());
  return U.data;
}

size_t differ(const std::vector<double>& a, const std::vector<double>& b) {
  size_t n = 0;
  for (size_t q = 0; q < a.size(); q++)
    if (!(a[q] == b[q]) && !(std::isnan(a[q]) && std::isnan(b[q]))) n++;
  return n;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s scheme(1|2|3) problem(ot|bw|dir) steps\n", argv[0]);
    return 2;
  }
  const int scheme = std::atoi(argv[1]), steps = std::atoi(argv[3]);
  const Problem p = make(argv[2]);
  double dA, dB, dC;
  std::vector<double> cA, cB, cC;
  const auto A = run(p, scheme, REF, steps, &dA, &cA);
  const auto B = run(p, scheme, REF_STEPPER_CUDA_METHOD, steps, &dB, &cB);
  const auto C = run(p, scheme, CUDA, steps, &dC, &cC);
  const size_t ab = differ(A, B), ac = differ(A, C), chb = differ(cA, cB), chc = differ(cA, cC);
  std::printf("%s scheme %d steps %d: ref-stepper+cuda-method %zu diffs (chars %zu, dt %s), "
              "cuda-stepper %zu diffs (chars %zu, dt %s)\n",
              argv[2], scheme, steps, ab, chb, dA == dB ? "same" : "DIFF", ac, chc,
              dA == dC ? "same" : "DIFF");
  return (ab || ac || chb || chc || dA != dB || dA != dC) ? 1 : 0;
}
