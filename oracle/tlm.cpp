// ORACLE — TEST INFRASTRUCTURE ONLY.  Tangent-linear (forward-mode)
// derivative of the oracle's discrete time stepping, the reference against
// which the CUDA discrete adjoint is checked.
//
// The C restatement (mhd_oracle.c) is compiled with a dual-number scalar:
// every value carries NT directional derivatives.  Comparisons look at the
// value only, so every branch (ENO stencils, upwinding, clamps, the dt
// ladder of updateDt, the RK3 retry rule) takes the same path as the plain
// run — the frozen-branch derivative.  dt only moves by powers of two from
// dt0, so its tangent stays zero: the dt sequence is frozen as well.  The
// Dirichlet edge snapshot is taken from the initial state inside the run
// (orc_run), so it carries the initial state's tangents.  The derivative
// of sqrt at 0 is taken as 0 (the one-sided convention of the adjoint).
// J = sum over the final interior of |m|^2 / (2 rho) dx dy.
#include <cmath>
#include <cstdlib>
#include <cstring>

constexpr int NT = 17;

struct Dual {
  double v;
  double d[NT];
  Dual() = default;
  Dual(double x) : v(x) {
    for (int q = 0; q < NT; q++) d[q] = 0.0;
  }
  explicit operator double() const { return v; }
};

static inline Dual lin(double v, const Dual& a, double ca, const Dual& b, double cb) {
  Dual r;
  r.v = v;
  for (int q = 0; q < NT; q++) r.d[q] = ca * a.d[q] + cb * b.d[q];
  return r;
}
static inline Dual operator+(const Dual& a, const Dual& b) { return lin(a.v + b.v, a, 1.0, b, 1.0); }
static inline Dual operator-(const Dual& a, const Dual& b) { return lin(a.v - b.v, a, 1.0, b, -1.0); }
static inline Dual operator*(const Dual& a, const Dual& b) { return lin(a.v * b.v, a, b.v, b, a.v); }
static inline Dual operator/(const Dual& a, const Dual& b) {
  const double r = a.v / b.v;
  return lin(r, a, 1.0 / b.v, b, -r / b.v);
}
static inline Dual operator-(const Dual& a) {
  Dual r;
  r.v = -a.v;
  for (int q = 0; q < NT; q++) r.d[q] = -a.d[q];
  return r;
}
static inline Dual operator+(const Dual& a) { return a; }
static inline Dual& operator+=(Dual& a, const Dual& b) { a = a + b; return a; }
static inline Dual& operator-=(Dual& a, const Dual& b) { a = a - b; return a; }
static inline Dual& operator*=(Dual& a, const Dual& b) { a = a * b; return a; }
static inline Dual& operator/=(Dual& a, const Dual& b) { a = a / b; return a; }
static inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
static inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
static inline bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
static inline bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
static inline bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
static inline bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }
static inline Dual sqrt(const Dual& a) {
  const double s = std::sqrt(a.v);
  Dual r;
  r.v = s;
  const double c = a.v > 0.0 ? 0.5 / s : 0.0;
  for (int q = 0; q < NT; q++) r.d[q] = c * a.d[q];
  return r;
}
static inline Dual fabs(const Dual& a) { return a.v < 0.0 ? -a : a; }
static inline Dual cos(const Dual& a) {
  Dual r;
  r.v = std::cos(a.v);
  const double c = -std::sin(a.v);
  for (int q = 0; q < NT; q++) r.d[q] = c * a.d[q];
  return r;
}
static inline bool isnan(const Dual& a) { return std::isnan(a.v); }

#define double Dual
extern "C" {
#include "mhd_oracle.c"
}
#undef double

extern "C" {

/* Runs nsteps steps (orc_run, no SOR) from U0 with ndir <= NT tangent
   directions dU0[r][8][NX][NY]; returns J, dJ[r] = dJ/dU0 . dU0[r], the
   final state and the step count. */
int tlm_run(int scheme, int time_method, int nx, int ny, double dx, double dy, double gamma,
            const int* bc, double dt_min, double dt_max, double cfl, int nsteps, double dt0,
            const double* U0, int ndir, const double* dU0, double* J, double* dJ, double* Uout,
            int* steps_done) {
  if (ndir < 0 || ndir > NT) return -1;
  const int NX = nx + 4, NY = ny + 4;
  const size_t tot = (size_t)8 * NX * NY;
  Dual* U = (Dual*)std::calloc(tot, sizeof(Dual));
  for (size_t q = 0; q < tot; q++) {
    U[q] = Dual(U0[q]);
    for (int r = 0; r < ndir; r++) U[q].d[r] = dU0[(size_t)r * tot + q];
  }
  orc_ctx* c = orc_create(scheme, time_method, nx, ny, dx, dy, gamma, bc, dt_min, dt_max, cfl);
  Dual dt = dt0, t = 0.0;
  int steps = 0, err = 0;
  const int st = orc_run(c, nsteps, 0.0, nullptr, 0, U, &dt, &t, &steps, nullptr, nullptr, 0, &err);
  Dual s = 0.0;
  for (int i = 2; i < nx + 2; i++)
    for (int j = 2; j < ny + 2; j++) {
      const Dual r = U[((size_t)0 * NX + i) * NY + j], mx = U[((size_t)1 * NX + i) * NY + j],
                 my = U[((size_t)2 * NX + i) * NY + j], mz = U[((size_t)3 * NX + i) * NY + j];
      s += Dual(0.5) * (mx * mx + my * my + mz * mz) / r;
    }
  s = s * (Dual(dx) * Dual(dy));
  *J = s.v;
  for (int r = 0; r < ndir; r++) dJ[r] = s.d[r];
  if (Uout)
    for (size_t q = 0; q < tot; q++) Uout[q] = U[q].v;
  if (steps_done) *steps_done = steps;
  orc_destroy(c);
  std::free(U);
  return st;
}

}  // extern "C"
