// ORACLE — test infrastructure only. Nothing in the shipped library links, calls or loads this
// file; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it, and only
// as the checker.
//
// A float64 CPU restatement of the reference's own CPU hydro scheme, src/reference/hydro.ts
// (RefHydro), and of its exact Riemann solver, src/reference/riemann_exact.ts. The structure
// follows the reference function by function (citations inline), in the same gather form:
// primitives -> dt -> memoised per-cell predictor -> per-face Riemann fluxes -> update.
//
// One extension has no counterpart in the reference: `recon = 4` (PPM), the Colella & Woodward
// (1984) parabolic interface values (their eqs. 1.6-1.10), used as the edge increments of the
// same MUSCL-Hancock predictor. Its parity is unpinned: no reference code exists for it.
//
// Pins: the exact solver reproduces the reference test's Toro values, the limiter identities
// and the scheme's convergence / conservation / symmetry properties (tests/test_oracle.py ports
// tests/unit/reference.test.ts case by case).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "hydro_ref.h"

namespace {

using namespace oracle;

// Colella & Woodward (1984): the parabola's edge values for the cell `c` given the five cells
// c-2..c+2 along one axis (eq. 1.6 with the limited slopes of eq. 1.8, then the monotonicity
// constraints of eq. 1.10). Returns the lower and upper edge values. Not in the reference.
inline double ppm_slope(double am, double a, double ap) {
  const double d = 0.5 * (ap - am);
  if ((ap - a) * (a - am) > 0)
    return sgn(d) * std::min(std::fabs(d), std::min(2 * std::fabs(a - am), 2 * std::fabs(ap - a)));
  return 0.0;
}
void ppm_edges(double a2m, double am, double a, double ap, double a2p, double* lo, double* hi) {
  const double dm = ppm_slope(a2m, am, a), d0 = ppm_slope(am, a, ap), dp = ppm_slope(a, ap, a2p);
  double al = 0.5 * (am + a) - (d0 - dm) / 6.0;
  double ar = 0.5 * (a + ap) - (dp - d0) / 6.0;
  if ((ar - a) * (a - al) <= 0) {
    al = a; ar = a;
  } else {
    const double da = ar - al, a6 = 6.0 * (a - 0.5 * (al + ar));
    if (da * a6 > da * da) al = 3 * a - 2 * ar;
    else if (-da * da > da * a6) ar = 3 * a - 2 * al;
  }
  *lo = al; *hi = ar;
}

struct Pred {
  double q[NQ];
  double su[3][NQ];
  double sd[3][NQ];
  double flag;
  bool first_order;
};

}  // namespace

extern "C" {

typedef struct orc_config {
  int32_t n[3];
  double dx;
  double gamma;
  int32_t bc_lo[3];
  int32_t bc_hi[3];
  double cfl;
  double rho_floor;
  double p_floor;
  double eta_dual;
  double shock_thresh;
  int32_t riemann;      // 0 hllc, 1 hll
  int32_t recon;        // 0 minmod, 1 mc, 2 vanleer, 3 koren, 4 ppm (extension)
  int32_t isentropic;   // hydro.ts RefConfig.isentropic
  int32_t signal_dims;  // the multiple of cs in the signal rate: 3 in hydro.ts:254
} orc_config;

}  // extern "C"

namespace {

struct Hydro {
  orc_config c;
  int64_t ncell;
  std::vector<double> U[7];  // rho, mx, my, mz, E, e_int, rho*s   (hydro.ts:175-176)
  std::vector<double> W;     // per cell: rho, vx, vy, vz, p, s, cs (hydro.ts:180)
  std::vector<Pred> preds;
  double t = 0, dt = 0;
  int64_t steps = 0;
  int threads = 1;

  int64_t index(int i, int j, int k) const { return ((int64_t)k * c.n[1] + j) * c.n[0] + i; }

  // hydro.ts:216-220 bcAxis: source index and velocity sign for a possibly out-of-range index.
  static void bc_axis(int i, int n, int lo, int hi, int* src, double* f) {
    if (i < 0) {
      if (lo == 0) { *src = ((i % n) + n) % n; *f = 1; }
      else if (lo == 1) { *src = 0; *f = 1; }
      else { *src = -1 - i; *f = -1; }
      return;
    }
    if (i >= n) {
      if (hi == 0) { *src = i % n; *f = 1; }
      else if (hi == 1) { *src = n - 1; *f = 1; }
      else { *src = 2 * n - 1 - i; *f = -1; }
      return;
    }
    *src = i; *f = 1;
  }

  // hydro.ts:223-231 loadQ.
  void load_q(int i, int j, int k, double* out) const {
    int x, y, z; double fx, fy, fz;
    bc_axis(i, c.n[0], c.bc_lo[0], c.bc_hi[0], &x, &fx);
    bc_axis(j, c.n[1], c.bc_lo[1], c.bc_hi[1], &y, &fy);
    bc_axis(k, c.n[2], c.bc_lo[2], c.bc_hi[2], &z, &fz);
    const double* w = &W[index(x, y, z) * 7];
    out[0] = w[0]; out[1] = w[1] * fx; out[2] = w[2] * fy; out[3] = w[3] * fz;
    out[4] = w[4]; out[5] = w[5]; out[6] = w[6];
  }

  // hydro.ts:233-257 primitives(); returns the largest signal rate.
  double primitives() {
    const double g = c.gamma;
    double rate = 0;
#pragma omp parallel for reduction(max : rate) num_threads(threads) schedule(static)
    for (int64_t o = 0; o < ncell; o++) {
      const double rho = std::max(U[0][o], c.rho_floor);
      double eint = U[5][o];
      double p = (g - 1) * eint;
      if (!(p >= c.p_floor)) { p = c.p_floor; eint = p / (g - 1); }
      const double cs = std::sqrt(g * p / rho);
      double* w = &W[o * 7];
      w[0] = rho; w[1] = U[1][o] / rho; w[2] = U[2][o] / rho; w[3] = U[3][o] / rho;
      w[4] = p; w[5] = U[6][o] / rho; w[6] = cs;
      rate = std::max(rate, std::fabs(w[1]) + std::fabs(w[2]) + std::fabs(w[3]) + c.signal_dims * cs);
    }
    return rate;
  }

  // hydro.ts:260-265 isen.
  void isen(double* out, const double* m, const double* q, const double* p, bool up) const {
    if (!c.isentropic || c.recon == PPM) return;
    double inc, b;
    isen_inc(m, q, p, out[4], up, c.recon, c.gamma, &inc, &b);
    out[0] += std::min(std::max(inc - out[0], -b), b);
  }

  // hydro.ts:268-270 scales.
  static void scales(const double* q, double* s) {
    s[0] = q[0]; s[1] = q[6]; s[2] = q[6]; s[3] = q[6]; s[4] = q[4]; s[5] = 0;
  }

  // The edge increments along axis a of the cell at (i, j, k), as hydro.ts:282-293 (the slope
  // limiters) and :347-356 (a ghost's recomputed edges); PPM (extension) reads two cells each way.
  void edges(int i, int j, int k, int a, const double* w, const double* scale, double* su, double* sd) const {
    const int e[3] = {a == 0, a == 1, a == 2};
    double m[7], p[7];
    load_q(i - e[0], j - e[1], k - e[2], m);
    load_q(i + e[0], j + e[1], k + e[2], p);
    if (c.recon == PPM) {
      double m2[7], p2[7];
      load_q(i - 2 * e[0], j - 2 * e[1], k - 2 * e[2], m2);
      load_q(i + 2 * e[0], j + 2 * e[1], k + 2 * e[2], p2);
      for (int v = 0; v < NQ; v++) {
        double lo, hi;
        ppm_edges(m2[v], m[v], w[v], p[v], p2[v], &lo, &hi);
        su[v] = 2 * (hi - w[v]);
        sd[v] = 2 * (w[v] - lo);
      }
      return;
    }
    for (int v = 0; v < NQ; v++) su[v] = limiter(c.recon, w[v] - m[v], p[v] - w[v], scale[v]);
    isen(su, m, w, p, true);
    for (int v = 0; v < NQ; v++) sd[v] = limiter(c.recon, p[v] - w[v], w[v] - m[v], scale[v]);
    isen(sd, m, w, p, false);
  }

  // hydro.ts:272-322 predictRaw.
  void predict_raw(int i, int j, int k, Pred* out) const {
    double q[7];
    load_q(i, j, k, q);
    double nb[3][2][7];
    load_q(i - 1, j, k, nb[0][0]); load_q(i + 1, j, k, nb[0][1]);
    load_q(i, j - 1, k, nb[1][0]); load_q(i, j + 1, k, nb[1][1]);
    load_q(i, j, k - 1, nb[2][0]); load_q(i, j, k + 1, nb[2][1]);
    double scale[NQ];
    scales(q, scale);
    for (int a = 0; a < 3; a++) edges(i, j, k, a, q, scale, out->su[a], out->sd[a]);
    double s[3][NQ];
    for (int a = 0; a < 3; a++)
      for (int v = 0; v < NQ; v++) s[a][v] = 0.5 * (out->su[a][v] + out->sd[a][v]);
    double big = -std::numeric_limits<double>::infinity();
    for (int a = 0; a < 3; a++) big = std::max(big, std::max(std::fabs(out->su[a][4]), std::fabs(out->sd[a][4])));
    double fall = 0;
    for (int a = 0; a < 3; a++) fall = std::min(fall, 0.5 * out->su[a][0]);
    for (int a = 0; a < 3; a++) fall = std::min(fall, -0.5 * out->sd[a][0]);
    const double conv = nb[0][1][1] - nb[0][0][1] + (nb[1][1][2] - nb[1][0][2]) + (nb[2][1][3] - nb[2][0][3]);
    double jump = -std::numeric_limits<double>::infinity();
    for (int a = 0; a < 3; a++)
      jump = std::max(jump, std::fabs(nb[a][1][4] - nb[a][0][4]) / std::min(nb[a][1][4], nb[a][0][4]));
    out->flag = (conv < 0 && jump > c.shock_thresh) ? 1.0 : 0.0;

    const double h = (0.5 * dt) / c.dx;
    const double rho = q[0], v[3] = {q[1], q[2], q[3]}, cs = q[6];
    const double dv = s[0][1] + s[1][2] + s[2][3];
    auto adv = [&](int n) { return v[0] * s[0][n] + v[1] * s[1][n] + v[2] * s[2][n]; };
    double qh[NQ];
    qh[0] = rho - h * (adv(0) + rho * dv);
    for (int d = 0; d < 3; d++) qh[1 + d] = v[d] - h * (adv(1 + d) + s[d][4] / rho);
    qh[4] = q[4] - h * (adv(4) + rho * cs * cs * dv);
    qh[5] = q[5] - h * adv(5);
    const double rmin = qh[0] + fall;
    const double pmin = qh[4] - 0.5 * big;
    if (!(rmin > 0 && pmin > 0)) {
      for (int n = 0; n < NQ; n++) out->q[n] = q[n];
      std::memset(out->su, 0, sizeof(out->su));
      std::memset(out->sd, 0, sizeof(out->sd));
      out->first_order = true;
      return;
    }
    for (int n = 0; n < NQ; n++) out->q[n] = qh[n];
    out->first_order = false;
  }

  // hydro.ts:329-358 predict: a cell in range is memoised; a cell beyond a boundary takes the
  // half-step state and flags of the cell it maps to (mirrored), with edges recomputed there.
  void predict(int i, int j, int k, Pred* out) const {
    if (i >= 0 && j >= 0 && k >= 0 && i < c.n[0] && j < c.n[1] && k < c.n[2]) {
      *out = preds[index(i, j, k)];
      return;
    }
    int x, y, z; double fx, fy, fz;
    bc_axis(i, c.n[0], c.bc_lo[0], c.bc_hi[0], &x, &fx);
    bc_axis(j, c.n[1], c.bc_lo[1], c.bc_hi[1], &y, &fy);
    bc_axis(k, c.n[2], c.bc_lo[2], c.bc_hi[2], &z, &fz);
    Pred src;
    predict(x, y, z, &src);
    for (int n = 0; n < NQ; n++) out->q[n] = src.q[n];
    out->q[1] *= fx; out->q[2] *= fy; out->q[3] *= fz;
    double w[7];
    load_q(i, j, k, w);
    double scale[NQ];
    scales(w, scale);
    for (int a = 0; a < 3; a++) {
      if (src.first_order) {
        for (int n = 0; n < NQ; n++) { out->su[a][n] = 0; out->sd[a][n] = 0; }
      } else {
        edges(i, j, k, a, w, scale, out->su[a], out->sd[a]);
      }
    }
    out->flag = src.flag;
    out->first_order = src.first_order;
  }

  // hydro.ts:360-375 side.
  Side side(const Pred& pr, int axis, int sg) const {
    const double g = c.gamma;
    auto f = [&](int n) { return pr.q[n] + 0.5 * sg * (sg > 0 ? pr.su : pr.sd)[axis][n]; };
    Side s;
    s.rho = std::max(f(0), c.rho_floor);
    s.p = std::max(f(4), c.p_floor);
    const double v[3] = {f(1), f(2), f(3)};
    s.v[0] = v[axis]; s.v[1] = v[(axis + 1) % 3]; s.v[2] = v[(axis + 2) % 3];
    s.s = f(5);
    s.cs = std::sqrt(g * s.p / s.rho);
    s.eint = s.p / (g - 1);
    return s;
  }

  // hydro.ts:378-452 step.
  double step(double t_end) {
    const double rate = primitives();
    dt = std::min((c.cfl * c.dx) / rate, std::max(t_end - t, 0.0));
    preds.resize(ncell);
#pragma omp parallel for collapse(2) num_threads(threads) schedule(static)
    for (int k = 0; k < c.n[2]; k++)
      for (int j = 0; j < c.n[1]; j++)
        for (int i = 0; i < c.n[0]; i++) predict_raw(i, j, k, &preds[index(i, j, k)]);
    const double dtdx = dt / c.dx;
    const double g = c.gamma;
    std::vector<double> next[7];
    for (int v = 0; v < 7; v++) next[v] = U[v];
    static const int OFF[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
#pragma omp parallel for collapse(2) num_threads(threads) schedule(static)
    for (int k = 0; k < c.n[2]; k++)
      for (int j = 0; j < c.n[1]; j++)
        for (int i = 0; i < c.n[0]; i++) {
          const int64_t o = index(i, j, k);
          const Pred& self = preds[o];
          double dm = 0, dmom[3] = {0, 0, 0}, de = 0, dei = 0, ds = 0, dvn = 0;
          for (int f = 0; f < 6; f++) {
            const int axis = f >> 1;
            const bool upper = (f & 1) == 1;
            // an in-range neighbour's memoised prediction is read in place; a ghost's is formed
            const int ni = i + OFF[f][0], nj = j + OFF[f][1], nk = k + OFF[f][2];
            Pred ghost;
            const bool inside = ni >= 0 && nj >= 0 && nk >= 0 && ni < c.n[0] && nj < c.n[1] && nk < c.n[2];
            if (!inside) predict(ni, nj, nk, &ghost);
            const Pred& nb = inside ? preds[index(ni, nj, nk)] : ghost;
            const Side L = upper ? side(self, axis, 1) : side(nb, axis, 1);
            const Side R = upper ? side(nb, axis, -1) : side(self, axis, -1);
            const double w = std::max(self.flag, nb.flag);
            const Flux F = riemann_flux(L, R, w, c.riemann == 1);
            const double sg = upper ? -1.0 : 1.0;
            dm += sg * F.m;
            for (int d = 0; d < 3; d++) dmom[(axis + d) % 3] += sg * F.mom[d];
            de += sg * F.e;
            dei += sg * F.ei;
            ds += sg * F.s;
            dvn += sg * F.vn;
          }
          const double rho = std::max(U[0][o] + dtdx * dm, c.rho_floor);
          double mom[3];
          for (int d = 0; d < 3; d++) mom[d] = U[1 + d][o] + dtdx * dmom[d];
          double E = U[4][o] + dtdx * de;
          double eint = U[5][o] + dtdx * (dei + std::max(self.q[4], c.p_floor) * dvn);
          const double ke = (0.5 * (mom[0] * mom[0] + mom[1] * mom[1] + mom[2] * mom[2])) / rho;
          const double eth = E - ke;
          const double emin = c.p_floor / (g - 1);
          if (eth > c.eta_dual * E && eth >= emin) {
            eint = eth;
          } else {
            if (!(eint >= emin)) eint = emin;
            E = ke + eint;
          }
          next[0][o] = rho;
          next[1][o] = mom[0]; next[2][o] = mom[1]; next[3][o] = mom[2];
          next[4][o] = E;
          next[5][o] = eint;
          next[6][o] = U[6][o] + dtdx * ds;
        }
    for (int v = 0; v < 7; v++) U[v].swap(next[v]);
    t += dt;
    steps++;
    return dt;
  }
};

}  // namespace

extern "C" {

void* orc_create(const orc_config* cfg) {
  Hydro* h = new Hydro();
  h->c = *cfg;
  h->ncell = (int64_t)cfg->n[0] * cfg->n[1] * cfg->n[2];
  for (int v = 0; v < 7; v++) h->U[v].assign(h->ncell, 0.0);
  h->W.assign(h->ncell * 7, 0.0);
  return h;
}

void orc_destroy(void* p) { delete static_cast<Hydro*>(p); }

void orc_set_threads(void* p, int n) { static_cast<Hydro*>(p)->threads = n < 1 ? 1 : n; }

// hydro.ts:195-214 init, from primitives given per cell as (rho, vx, vy, vz, p, s), x fastest.
void orc_init_prims(void* p, const double* prims) {
  Hydro* h = static_cast<Hydro*>(p);
  const double g = h->c.gamma;
  for (int64_t o = 0; o < h->ncell; o++) {
    const double* w = prims + o * 6;
    const double rho = w[0], eint = w[4] / (g - 1);
    h->U[0][o] = rho;
    h->U[1][o] = rho * w[1];
    h->U[2][o] = rho * w[2];
    h->U[3][o] = rho * w[3];
    h->U[4][o] = eint + 0.5 * rho * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
    h->U[5][o] = eint;
    h->U[6][o] = rho * w[5];
  }
  h->t = 0;
  h->steps = 0;
}

// Conserved state as 7 planes of ncell doubles: rho, mx, my, mz, E, e_int, rho*s.
void orc_set_conserved(void* p, const double* u) {
  Hydro* h = static_cast<Hydro*>(p);
  for (int v = 0; v < 7; v++) std::memcpy(h->U[v].data(), u + v * h->ncell, sizeof(double) * h->ncell);
}
void orc_get_conserved(void* p, double* u) {
  Hydro* h = static_cast<Hydro*>(p);
  for (int v = 0; v < 7; v++) std::memcpy(u + v * h->ncell, h->U[v].data(), sizeof(double) * h->ncell);
}

double orc_step(void* p, double t_end) { return static_cast<Hydro*>(p)->step(t_end); }

// hydro.ts:455-457 run.
void orc_run(void* p, double t_end, int64_t max_steps) {
  Hydro* h = static_cast<Hydro*>(p);
  while (h->t < t_end * (1 - 1e-12) && h->steps < max_steps) h->step(t_end);
}

double orc_time(void* p) { return static_cast<Hydro*>(p)->t; }
double orc_dt(void* p) { return static_cast<Hydro*>(p)->dt; }
int64_t orc_steps(void* p) { return static_cast<Hydro*>(p)->steps; }
void orc_set_clock(void* p, double t, int64_t steps) {
  Hydro* h = static_cast<Hydro*>(p);
  h->t = t;
  h->steps = steps;
}

double orc_limiter(int kind, double a, double b, double scale) { return limiter(kind, a, b, scale); }

void orc_ppm_edges(double a2m, double am, double a, double ap, double a2p, double* lo, double* hi) {
  ppm_edges(a2m, am, a, ap, a2p, lo, hi);
}

// riemann_exact.ts:9-71 exactRiemann: samples (rho, u, p) at each xi = x / t.
void orc_exact_riemann(double rl, double ul, double pl, double rr, double ur, double pr, double g,
                       const double* xi, int64_t n, double* out) {
  const double cL = std::sqrt(g * pl / rl), cR = std::sqrt(g * pr / rr);
  auto fK = [&](double p, double rho, double ps, double c, double* f, double* df) {
    if (p > ps) {
      const double A = 2 / ((g + 1) * rho), B = ((g - 1) / (g + 1)) * ps;
      const double q = std::sqrt(A / (p + B));
      *f = (p - ps) * q;
      *df = q * (1 - (p - ps) / (2 * (B + p)));
      return;
    }
    const double r = p / ps;
    *f = ((2 * c) / (g - 1)) * (std::pow(r, (g - 1) / (2 * g)) - 1);
    *df = (1 / (rho * c)) * std::pow(r, -(g + 1) / (2 * g));
  };
  const double z = (g - 1) / (2 * g);
  double p = std::pow((cL + cR - 0.5 * (g - 1) * (ur - ul)) / (cL / std::pow(pl, z) + cR / std::pow(pr, z)), 1 / z);
  p = std::max(p, 1e-12);
  for (int i = 0; i < 100; i++) {
    double fl, dl, fr, dr;
    fK(p, rl, pl, cL, &fl, &dl);
    fK(p, rr, pr, cR, &fr, &dr);
    const double pn = std::max(p - (fl + fr + ur - ul) / (dl + dr), 1e-14);
    const double change = (2 * std::fabs(pn - p)) / (pn + p);
    p = pn;
    if (change < 1e-14) break;
  }
  const double ps = p;
  double fl, dl, fr, dr;
  fK(ps, rr, pr, cR, &fr, &dr);
  fK(ps, rl, pl, cL, &fl, &dl);
  const double us = 0.5 * (ul + ur) + 0.5 * (fr - fl);
  const double gm = (g - 1) / (g + 1);
  for (int64_t i = 0; i < n; i++) {
    const double x = xi[i];
    double* o = out + 3 * i;
    auto put = [&](double a, double b, double c) { o[0] = a; o[1] = b; o[2] = c; };
    if (x <= us) {
      if (ps > pl) {
        const double sL = ul - cL * std::sqrt(((g + 1) / (2 * g)) * (ps / pl) + (g - 1) / (2 * g));
        if (x <= sL) put(rl, ul, pl);
        else put((rl * (ps / pl + gm)) / (gm * (ps / pl) + 1), us, ps);
        continue;
      }
      const double head = ul - cL, cs = cL * std::pow(ps / pl, z), tail = us - cs;
      if (x <= head) { put(rl, ul, pl); continue; }
      if (x >= tail) { put(rl * std::pow(ps / pl, 1 / g), us, ps); continue; }
      const double cc = (2 / (g + 1)) * (cL + 0.5 * (g - 1) * (ul - x));
      put(rl * std::pow(cc / cL, 2 / (g - 1)), (2 / (g + 1)) * (cL + 0.5 * (g - 1) * ul + x),
          pl * std::pow(cc / cL, (2 * g) / (g - 1)));
      continue;
    }
    if (ps > pr) {
      const double sR = ur + cR * std::sqrt(((g + 1) / (2 * g)) * (ps / pr) + (g - 1) / (2 * g));
      if (x >= sR) put(rr, ur, pr);
      else put((rr * (ps / pr + gm)) / (gm * (ps / pr) + 1), us, ps);
      continue;
    }
    const double head = ur + cR, cs = cR * std::pow(ps / pr, z), tail = us + cs;
    if (x >= head) { put(rr, ur, pr); continue; }
    if (x <= tail) { put(rr * std::pow(ps / pr, 1 / g), us, ps); continue; }
    const double cc = (2 / (g + 1)) * (cR - 0.5 * (g - 1) * (ur - x));
    put(rr * std::pow(cc / cR, 2 / (g - 1)), (2 / (g + 1)) * (-cR + 0.5 * (g - 1) * ur + x),
        pr * std::pow(cc / cR, (2 * g) / (g - 1)));
  }
}

}  // extern "C"
