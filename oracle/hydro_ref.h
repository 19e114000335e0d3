// ORACLE — test infrastructure only (see ref_hydro.cpp). The float64 arithmetic of one cell and
// one face of the reference's CPU scheme (src/reference/hydro.ts), shared by the uniform-grid
// oracle (ref_hydro.cpp) and the block-grid oracle (amr_ref.cpp).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>

namespace oracle {

enum Recon { MINMOD = 0, MC = 1, VANLEER = 2, KOREN = 3, PPM = 4 };
constexpr int NQ = 6;  // primitive vector: rho, vx, vy, vz, p, s

inline double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }

// hydro.ts:29 KOREN_SMOOTH, :30-46 LIMITERS. (far, near, scale) -> edge increment.
constexpr double KOREN_SMOOTH = 0.01;
inline double limiter(int kind, double a, double b, double scale) {
  switch (kind) {
    case MC:
      return a * b > 0 ? sgn(a) * std::min(std::min(2 * std::fabs(a), 2 * std::fabs(b)), 0.5 * std::fabs(a + b)) : 0.0;
    case VANLEER:
      return a * b > 0 ? (2 * a * b) / (a + b) : 0.0;
    case MINMOD:
      return a * b > 0 ? sgn(a) * std::min(std::fabs(a), std::fabs(b)) : 0.0;
    case KOREN: {
      const double far = a, near = b;
      const double fr = (far + 2 * near) / 3;
      const double lim = far * near > 0
          ? sgn(near) * std::min(std::min(2 * std::fabs(far), 2 * std::fabs(near)), std::fabs(fr))
          : 0.0;
      const double s = KOREN_SMOOTH * scale;
      const bool as_is = (s * s >= 1e-30 && s * s < 1e30) || s == 0;
      const double eta = as_is ? (far * far + near * near) / std::max(s * s, 1e-30)
                               : std::pow(far / std::fabs(s), 2) + std::pow(near / std::fabs(s), 2);
      const double w = std::min(std::max(1.5 - eta, 0.0), 1.0);
      return lim + (fr - lim) * w;
    }
    default:
      return 0.0;
  }
}

// hydro.ts:49-56 ISEN_* constants.
constexpr double ISEN_SMOOTH = 0.2, ISEN_ADIABAT = 0.01, ISEN_SHEAR = 0.1, ISEN_CAP = 0.25, ISEN_ROOM = 0.01;

// hydro.ts:65-83 isenInc. m, q, p: [rho, vx, vy, vz, p, s, cs] of the lower neighbour, the cell
// and the upper neighbour. Returns (twice the increment along the adiabat, its bound).
inline void isen_inc(const double* m, const double* q, const double* p, double p_inc, bool up, int lim_kind,
              double gamma, double* inc, double* bound) {
  const double rl = m[0], pl = m[4], rc = q[0], pc = q[4], rr = p[0], pr = p[4];
  if (!(rl > 0 && pl > 0 && rc > 0 && pc > 0 && rr > 0 && pr > 0)) { *inc = 0; *bound = 0; return; }
  const double gi = 1 / gamma;
  const double tl = rl * std::pow(pc / pl, gi) - rc;
  const double tr = rr * std::pow(pc / pr, gi) - rc;
  const double sg = up ? 1.0 : -1.0;
  const double d = up ? limiter(lim_kind, -tl, tr, rc) : limiter(lim_kind, tr, -tl, rc);
  const double pf = pc + 0.5 * sg * p_inc;
  const double rn = up ? rr : rl;
  const double rf = std::min(std::max((rc + 0.5 * sg * d) * std::pow(std::max(pf, 1e-30) / pc, gi), std::min(rc, rn)),
                             std::max(rc, rn));
  auto fade = [](double x) { return std::min(std::max(2 - x, 0.0), 1.0); };
  auto dv = [](const double* a, const double* b) {
    return std::hypot(std::hypot(a[1] - b[1], a[2] - b[2]), a[3] - b[3]);
  };
  const double ks = fade(std::max(std::fabs(pl - pc), std::fabs(pr - pc)) / (ISEN_SMOOTH * pc));
  const double ka = fade(std::max(std::fabs(tl), std::fabs(tr)) / (ISEN_ADIABAT * rc));
  const double kv = fade(std::max(dv(p, q), dv(q, m)) / (ISEN_SHEAR * std::max(q[6], 1e-30)));
  *bound = std::max(ISEN_CAP * std::min(std::fabs(rc - rl), std::fabs(rr - rc)), ISEN_ROOM * rc * ks * ka * kv);
  *inc = 2 * sg * (rf - rc);
}

struct Side { double rho, v[3], p, s, cs, eint; };
struct Flux { double m, mom[3], e, ei, s, vn; };

// hydro.ts:102-159 riemannFlux (HLLC with an HLL blend by w_hll; HLL when hll != 0).
inline Flux riemann_flux(const Side& l, const Side& r, double w_hll, bool hll) {
  const double sl = std::min(l.v[0] - l.cs, r.v[0] - r.cs);
  const double sr = std::max(l.v[0] + l.cs, r.v[0] + r.cs);
  auto ke = [](const Side& s) { return 0.5 * s.rho * (s.v[0] * s.v[0] + s.v[1] * s.v[1] + s.v[2] * s.v[2]); };
  const double el = l.eint + ke(l), er = r.eint + ke(r);
  double ml[3], mr[3], fpl[3], fpr[3];
  for (int i = 0; i < 3; i++) { ml[i] = l.rho * l.v[i]; mr[i] = r.rho * r.v[i]; }
  fpl[0] = ml[0] * l.v[0] + l.p; fpl[1] = ml[1] * l.v[0]; fpl[2] = ml[2] * l.v[0];
  fpr[0] = mr[0] * r.v[0] + r.p; fpr[1] = mr[1] * r.v[0]; fpr[2] = mr[2] * r.v[0];
  const double fel = (el + l.p) * l.v[0], fer = (er + r.p) * r.v[0];
  Flux F;
  if (sl >= 0) {
    F.m = ml[0]; for (int i = 0; i < 3; i++) F.mom[i] = fpl[i]; F.e = fel; F.vn = l.v[0];
  } else if (sr <= 0) {
    F.m = mr[0]; for (int i = 0; i < 3; i++) F.mom[i] = fpr[i]; F.e = fer; F.vn = r.v[0];
  } else {
    const double ql = l.rho * (sl - l.v[0]);
    const double qr = r.rho * (sr - r.v[0]);
    const double sm = (r.p - l.p + l.v[0] * ql - r.v[0] * qr) / (ql - qr);
    const double inv = 1 / (sr - sl);
    const double hm = (sr * ml[0] - sl * mr[0] + sl * sr * (r.rho - l.rho)) * inv;
    double hp[3];
    for (int i = 0; i < 3; i++) hp[i] = (sr * fpl[i] - sl * fpr[i] + sl * sr * (mr[i] - ml[i])) * inv;
    const double he = (sr * fel - sl * fer + sl * sr * (er - el)) * inv;
    double cm, cp[3], ce;
    if (sm >= 0) {
      const double f = ql / (sl - sm);
      const double ms[3] = {f * sm, f * l.v[1], f * l.v[2]};
      const double es = f * (el / l.rho + (sm - l.v[0]) * (sm + l.p / ql));
      cm = ml[0] + sl * (f - l.rho);
      for (int i = 0; i < 3; i++) cp[i] = fpl[i] + sl * (ms[i] - ml[i]);
      ce = fel + sl * (es - el);
    } else {
      const double f = qr / (sr - sm);
      const double ms[3] = {f * sm, f * r.v[1], f * r.v[2]};
      const double es = f * (er / r.rho + (sm - r.v[0]) * (sm + r.p / qr));
      cm = mr[0] + sr * (f - r.rho);
      for (int i = 0; i < 3; i++) cp[i] = fpr[i] + sr * (ms[i] - mr[i]);
      ce = fer + sr * (es - er);
    }
    const double w = hll ? 1.0 : w_hll;
    F.m = cm + (hm - cm) * w;
    for (int i = 0; i < 3; i++) F.mom[i] = cp[i] + (hp[i] - cp[i]) * w;
    F.e = ce + (he - ce) * w;
    F.vn = sm;
  }
  const bool up = F.m >= 0;
  F.ei = F.m * (up ? l.eint / l.rho : r.eint / r.rho);
  F.s = F.m * (up ? l.s : r.s);
  return F;
}

}  // namespace oracle
