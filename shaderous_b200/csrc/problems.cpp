// Host-side initial conditions of the built-in problems, in float64 at cell centres.
//
// Positions follow the reference: cell (i, j, k) is centred at (i + 0.5 - n/2) dx along each
// axis, the box centred on 0 (src/reference/hydro.ts:200, src/domain.ts:15). The primitives are
// (rho, vx, vy, vz, p, s); the caller rounds the conserved state to float32 once, as
// Sim.reset does (src/sim.ts:2704-2848).
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../include/shaderous_b200.h"
#include "problems.h"

namespace shz {

namespace {

constexpr double PI = 3.14159265358979323846;

// SplitMix64 (Steele, Lea & Flood 2014): a counter-based stream, so that the noise of a cell
// depends only on the seed and the cell's index, whatever slab of planes is generated.
inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
inline double unit_open(uint64_t x) { return ((x >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
// One standard normal deviate per cell (Box & Muller 1958).
inline double gauss(uint64_t seed, uint64_t cell) {
  const double u1 = unit_open(splitmix64(seed ^ (2 * cell)));
  const double u2 = unit_open(splitmix64(seed ^ (2 * cell + 1)));
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * PI * u2);
}

int ndim_of(const shz_config& c) { return c.n[2] > 1 ? 3 : (c.n[1] > 1 ? 2 : 1); }

// Sedov deposit, as src/setup/parts/region.ts:199-215: the energy is spread evenly over the cells
// whose centres lie inside the radius; returns that count.
int64_t sedov_count(const shz_config& c, double radius) {
  const int nd = ndim_of(c);
  const double dx = c.dx;
  const int reach = (int)std::ceil(radius / dx) + 1;
  int64_t count = 0;
  for (int k = (nd == 3 ? -reach : 0); k < (nd == 3 ? reach : 1); k++)
    for (int j = (nd >= 2 ? -reach : 0); j < (nd >= 2 ? reach : 1); j++)
      for (int i = -reach; i < reach; i++) {
        const double a = i + 0.5, b = nd >= 2 ? j + 0.5 : 0.0, d = nd == 3 ? k + 0.5 : 0.0;
        if (std::sqrt(a * a + b * b + d * d) * dx < radius) count++;
      }
  return count;
}

}  // namespace

ProblemCtx prepare_problem(const shz_config& c, const shz_problem& p) {
  ProblemCtx x;
  x.p = p;
  x.gamma = c.gamma;
  x.nd = ndim_of(c);
  x.L[0] = c.n[0] * c.dx;
  x.L[1] = c.n[1] * c.dx;
  x.L[2] = c.n[2] * c.dx;
  if (p.kind == SHZ_PROB_SEDOV) {
    x.sedov_r = p.a[3] * c.dx;
    const int64_t cnt = sedov_count(c, x.sedov_r);
    const double e_dep = p.a[2] / ((double)(cnt > 0 ? cnt : 1) * std::pow(c.dx, x.nd));
    x.sedov_p = (c.gamma - 1) * e_dep;
  }
  return x;
}

// The primitives (rho, vx, vy, vz, p, s) at a cell centre (x, y, z), box centred on 0; `cell`
// numbers the cell for the seeded noise.
void sample_problem(const ProblemCtx& q, double x, double y, double z, uint64_t cell, double* w) {
  const shz_problem& p = q.p;
  const int nd = q.nd;
  const double Lx = q.L[0], Ly = q.L[1], Lz = q.L[2];
  double rho = 1, vx = 0, vy = 0, vz = 0, pr = 1, s = 0;
  switch (p.kind) {
    case SHZ_PROB_SOD: {
      const double xn = p.axis == 0 ? x : (p.axis == 1 ? y : z);
      const bool left = xn < 0;
      rho = left ? p.a[0] : p.a[3];
      const double u = left ? p.a[1] : p.a[4];
      pr = left ? p.a[2] : p.a[5];
      (p.axis == 0 ? vx : (p.axis == 1 ? vy : vz)) = u;
      s = left ? 1 : 0;
      break;
    }
    case SHZ_PROB_KH: {
      // A dense slab |y - 1/2| < 1/4 of [0,1]^2 sliding through lighter gas; a seeded mode and
      // gaussian noise in vy (the kick of src/setup/parts/flows/kelvin_helmholtz.ts, with the
      // perturbation of the benchmark's own statement).
      const double X = x + Lx / 2, Y = y + Ly / 2;
      const bool inner = std::fabs(Y - 0.5 * Ly) < 0.25 * Ly;
      rho = inner ? p.a[0] : p.a[1];
      vx = inner ? p.a[2] : -p.a[2];
      vy = p.a[4] * std::sin(4 * PI * X / Lx) + p.a[5] * gauss(p.seed, cell);
      pr = p.a[3];
      s = inner ? 1 : 0;
      break;
    }
    case SHZ_PROB_TGV: {
      // On [0, 2 pi]^3 (box centred on 0, so shifted by half the box).
      const double X = (x + Lx / 2) * (2 * PI / Lx), Y = (y + Ly / 2) * (2 * PI / Ly), Z = (z + Lz / 2) * (2 * PI / Lz);
      rho = p.a[0];
      vx = p.a[2] * std::sin(X) * std::cos(Y) * std::cos(Z);
      vy = -p.a[2] * std::cos(X) * std::sin(Y) * std::cos(Z);
      vz = 0;
      pr = p.a[1];
      s = 0;
      break;
    }
    case SHZ_PROB_SEDOV: {
      const double r = std::sqrt(x * x + (nd >= 2 ? y * y : 0) + (nd == 3 ? z * z : 0));
      rho = p.a[0];
      pr = r < q.sedov_r ? q.sedov_p : p.a[1];
      s = r < q.sedov_r ? 1 : 0;
      break;
    }
    case SHZ_PROB_ADVECT: {
      const double X = x + Lx / 2;
      rho = p.a[0] + p.a[1] * std::sin(2 * PI * X / Lx);
      vx = p.a[2]; vy = p.a[3]; vz = p.a[4];
      pr = p.a[5];
      s = X < 0.5 * Lx ? 1 : 0;
      break;
    }
    case SHZ_PROB_BLAST: {
      const double r = std::sqrt(x * x + (nd >= 2 ? y * y : 0) + (nd == 3 ? z * z : 0));
      const bool in = r < p.a[4];
      rho = in ? p.a[0] : p.a[2];
      pr = in ? p.a[1] : p.a[3];
      s = in ? 1 : 0;
      break;
    }
    case SHZ_PROB_GAUSS: {
      const double r2 = x * x + y * y;
      rho = p.a[0] + std::exp(-r2 / p.a[1]);
      vx = p.a[2]; vy = p.a[3];
      vz = p.a[4] * std::sin(8 * PI * z);
      pr = p.a[5] + 0.5 * std::exp(-r2 / p.a[6]);
      s = 0;
      break;
    }
    default:
      break;
  }
  w[0] = rho; w[1] = vx; w[2] = vy; w[3] = vz; w[4] = pr; w[5] = s;
}

int problem_prims(const shz_config& c, const shz_problem& p, int k0, int k1, double* out) {
  const int nx = c.n[0], ny = c.n[1], nz = c.n[2];
  const double dx = c.dx;
  const ProblemCtx q = prepare_problem(c, p);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = k0; k < k1; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        const double x = (i + 0.5 - nx / 2.0) * dx, y = (j + 0.5 - ny / 2.0) * dx, z = (k + 0.5 - nz / 2.0) * dx;
        const uint64_t cell = ((uint64_t)k * ny + j) * nx + i;
        sample_problem(q, x, y, z, cell, out + ((int64_t)(k - k0) * ny * nx + (int64_t)j * nx + i) * 6);
      }
  return 0;
}

bool problem_known(int kind) { return kind >= SHZ_PROB_SOD && kind <= SHZ_PROB_GAUSS; }

void prims_to_state(const double* w, double gamma, int64_t count, float* u1, float* u2) {
#pragma omp parallel for schedule(static)
  for (int64_t o = 0; o < count; o++) {
    const double* q = w + o * 6;
    const double rho = q[0], eint = q[4] / (gamma - 1);
    const double ke = 0.5 * rho * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    u1[4 * o + 0] = (float)rho;
    u1[4 * o + 1] = (float)(rho * q[1]);
    u1[4 * o + 2] = (float)(rho * q[2]);
    u1[4 * o + 3] = (float)(rho * q[3]);
    u2[4 * o + 0] = (float)(eint + ke);
    u2[4 * o + 1] = (float)eint;
    u2[4 * o + 2] = (float)(rho * q[5]);
    u2[4 * o + 3] = 0.0f;
  }
}

}  // namespace shz

extern "C" int shz_problem_prims(const shz_config* cfg, const shz_problem* prob, int32_t k0, int32_t k1, double* prims) {
  if (!cfg || !prob || !prims) return SHZ_E_CONFIG;
  if (k0 < 0 || k1 > cfg->n[2] || k0 > k1) return SHZ_E_CONFIG;
  if (!shz::problem_known(prob->kind)) return SHZ_E_CONFIG;
  return shz::problem_prims(*cfg, *prob, k0, k1, prims);
}
