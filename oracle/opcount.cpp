// ORACLE — TEST INFRASTRUCTURE ONLY.  Floating-point operation count of the
// hot path, from the oracle restatement (mhd_oracle.c) compiled with a
// counting scalar type: +, -, *, /, sqrt count 1 each.  Divisions and square
// roots with a nonzero operand are also counted on their own (each costs a
// multi-instruction correctly rounded sequence on the GPU).
//
// Two counts are kept:
//   dense   — every operation the reference formulas perform as written;
//   nonzero — operations none of whose operands is an exact zero.  On a
//             state with no zero field (a seeded random state), the only
//             exact zeros are the structural ones (the dummy wave 7, the Bx
//             column, the zero entries of the Alfven rows, F[4] / G[5]), so
//             this is the algorithmic count the CUDA kernels perform.
// Prints one JSON object: counts per interior cell for one spatial operator
// (integrate) and one RK3 step, for ENO-Roe and ENO-LF.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

static unsigned long long g_dense = 0, g_nonzero = 0, g_div = 0, g_sqrt = 0;

struct CountedDouble {
  double v;
  CountedDouble() = default;
  CountedDouble(double x) : v(x) {}
  explicit operator double() const { return v; }
};
static inline bool operator<(CountedDouble a, CountedDouble b) { return a.v < b.v; }
static inline bool operator>(CountedDouble a, CountedDouble b) { return a.v > b.v; }
static inline bool operator<=(CountedDouble a, CountedDouble b) { return a.v <= b.v; }
static inline bool operator>=(CountedDouble a, CountedDouble b) { return a.v >= b.v; }
static inline bool operator==(CountedDouble a, CountedDouble b) { return a.v == b.v; }
static inline bool operator!=(CountedDouble a, CountedDouble b) { return a.v != b.v; }
static inline CountedDouble op(double r, double a, double b) {
  g_dense++;
  if (a != 0.0 && b != 0.0) g_nonzero++;
  return CountedDouble(r);
}
static inline CountedDouble operator+(CountedDouble a, CountedDouble b) { return op(a.v + b.v, a.v, b.v); }
static inline CountedDouble operator-(CountedDouble a, CountedDouble b) { return op(a.v - b.v, a.v, b.v); }
static inline CountedDouble operator*(CountedDouble a, CountedDouble b) { return op(a.v * b.v, a.v, b.v); }
static inline CountedDouble operator/(CountedDouble a, CountedDouble b) {
  if (a.v != 0.0) g_div++;
  return op(a.v / b.v, a.v, b.v);
}
static inline CountedDouble operator-(CountedDouble a) { return CountedDouble(-a.v); }
static inline CountedDouble operator+(CountedDouble a) { return a; }
static inline CountedDouble& operator+=(CountedDouble& a, CountedDouble b) { a = a + b; return a; }
static inline CountedDouble& operator-=(CountedDouble& a, CountedDouble b) { a = a - b; return a; }
static inline CountedDouble& operator*=(CountedDouble& a, CountedDouble b) { a = a * b; return a; }
static inline CountedDouble& operator/=(CountedDouble& a, CountedDouble b) { a = a / b; return a; }
static inline CountedDouble sqrt(CountedDouble a) {
  if (a.v != 0.0) g_sqrt++;
  return op(std::sqrt(a.v), a.v, 1.0);
}
static inline CountedDouble fabs(CountedDouble a) { return CountedDouble(std::fabs(a.v)); }
static inline CountedDouble cos(CountedDouble a) { return op(std::cos(a.v), a.v, 1.0); }
static inline bool isnan(CountedDouble a) { return std::isnan(a.v); }

#define double CountedDouble
extern "C" {
#include "mhd_oracle.c"
}
#undef double

static void random_state(double* U, int nx, int ny, double gm, unsigned seed) {
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> uni(-1.0, 1.0);
  const int NX = nx + 4, NY = ny + 4;
  for (int i = 2; i < nx + 2; i++)
    for (int j = 2; j < ny + 2; j++) {
      const double r = 1.0 + 0.2 * uni(rng), u = 0.3 * uni(rng), v = 0.3 * uni(rng),
                   w = 0.3 * uni(rng), bx = 0.8 + 0.2 * uni(rng), by = 0.5 + 0.2 * uni(rng),
                   bz = 0.3 + 0.2 * uni(rng), p = 1.0 + 0.2 * uni(rng);
      double* q[8];
      for (int k = 0; k < 8; k++) q[k] = &U[((size_t)k * NX + i) * NY + j];
      *q[0] = r; *q[1] = u * r; *q[2] = v * r; *q[3] = w * r;
      *q[4] = bx; *q[5] = by; *q[6] = bz;
      *q[7] = p / (gm - 1.0) + 0.5 * r * (u * u + v * v + w * w) + 0.5 * (bx * bx + by * by + bz * bz);
    }
}

int main(int argc, char** argv) {
  const int n = argc > 1 ? std::atoi(argv[1]) : 64;
  const double gm = 5.0 / 3.0, dx = 1.0 / n;
  const int bc[4] = {1, 1, 1, 1};
  const size_t tot = (size_t)8 * (n + 4) * (n + 4);
  std::printf("{\"cells\": %d", n * n);
  for (int scheme = 2; scheme <= 3; scheme++) {
    CountedDouble* U = (CountedDouble*)std::calloc(tot, sizeof(CountedDouble));
    CountedDouble* UL = (CountedDouble*)std::calloc(tot, sizeof(CountedDouble));
    double* Ud = (double*)std::calloc(tot, sizeof(double));
    random_state(Ud, n, n, gm, 12345u + scheme);
    for (size_t q = 0; q < tot; q++) U[q] = Ud[q];
    orc_ctx* c = orc_create(scheme, 2, n, n, dx, dx, gm, bc, 0.0, 1e-4, 0.0);
    CountedDouble ideal = 0.0, dt = 1e-4;
    int err = 0;
    g_dense = g_nonzero = g_div = g_sqrt = 0;
    orc_integrate(c, U, UL, &ideal, &err);
    const double id = double(g_dense) / (n * n), inz = double(g_nonzero) / (n * n);
    const double idiv = double(g_div) / (n * n), isq = double(g_sqrt) / (n * n);
    g_dense = g_nonzero = 0;
    orc_step(c, U, &dt, &err);
    const double sd = double(g_dense) / (n * n), snz = double(g_nonzero) / (n * n);
    std::printf(", \"%s\": {\"integrate_dense\": %.2f, \"integrate_nonzero\": %.2f, "
                "\"integrate_div\": %.2f, \"integrate_sqrt\": %.2f, "
                "\"step_dense\": %.2f, \"step_nonzero\": %.2f}",
                scheme == 2 ? "eno_roe" : "eno_lf", id, inz, idiv, isq, sd, snz);
    orc_destroy(c);
    std::free(U); std::free(UL); std::free(Ud);
  }
  std::printf("}\n");
  return 0;
}
