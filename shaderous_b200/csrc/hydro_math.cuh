// Float32 device arithmetic of one hydro step: limiters, the density along the adiabat, face
// states and the HLLC/HLL Riemann flux. Each function states the reference function it follows;
// the reference's CPU scheme is src/reference/hydro.ts, its shaders src/hydro/*.wgsl.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace shz {

enum Recon { R_MINMOD = 0, R_MC = 1, R_VANLEER = 2, R_KOREN = 3, R_PPM = 4 };

// Kernel parameters, passed by value.
struct KParams {
  double dx;  // cell size
  int n[3];
  int bc_lo[3], bc_hi[3];
  float gamma, gm1, inv_gm1, inv_gamma;
  float rho_floor, p_floor, e_floor;
  float eta_dual, shock_thresh, signal;
  int hll;
  double dv;  // cell volume dx^ndim in float64 (the float64 totals are scaled by it)
};

// The clock on the device (the reference's Clock, src/hydro/common.wgsl:84-96), advanced by
// clock_kernel before each sweep: t is the time of the state the sweep in flight produces.
struct DevClock {
  double t;
  double dt;
  double t_end;
  double dt_max;
  double cfl_dx;
  double last_dt;
  long long steps;
  long long max_steps;  // the clock holds once this many steps are taken (a batched request's length)
  int held;
  int bad;
};

// (Bitwise & and | rather than && and ||: no short-circuit, so no branch; the same values.)
__device__ __forceinline__ bool same_sign(float a, float b) { return ((a > 0.f) & (b > 0.f)) | ((a < 0.f) & (b < 0.f)); }

// hydro.ts:30-46 LIMITERS: the edge increment from the differences (far, near) and the
// quantity's natural scale (Koren only). The product test a*b > 0 is taken by signs, which is
// the same test without float32 underflow (as limiters/koren.wgsl:46-48 does).
template <int R>
__device__ __forceinline__ float limit(float a, float b, float scale) {
  if constexpr (R == R_MINMOD) {
    return same_sign(a, b) ? copysignf(fminf(fabsf(a), fabsf(b)), a) : 0.f;
  } else if constexpr (R == R_MC) {
    return same_sign(a, b) ? copysignf(fminf(fminf(2.f * fabsf(a), 2.f * fabsf(b)), 0.5f * fabsf(a + b)), a) : 0.f;
  } else if constexpr (R == R_VANLEER) {
    return same_sign(a, b) ? (2.f * a * b) / (a + b) : 0.f;
  } else {
    // Koren's limited third-order increment, unlimited where the change is small against the
    // scale (hydro.ts:35-45; SMOOTH = 0.01).
    const float far = a, near = b;
    const float fr = (far + 2.f * near) * (1.f / 3.f);
    const float lim = same_sign(far, near)
        ? copysignf(fminf(fminf(2.f * fabsf(far), 2.f * fabsf(near)), fabsf(fr)), near) : 0.f;
    const float s = 0.01f * scale;
    const float s2 = s * s;
    const bool as_is = ((s2 >= 1e-30f) & (s2 < 1e30f)) | (s == 0.f);
    // both forms, one kept (a select rather than a branch)
    const float eta_as_is = (far * far + near * near) / fmaxf(s2, 1e-30f);
    const float k = 1.f / fabsf(s);
    const float eta_scaled = (far * k) * (far * k) + (near * k) * (near * k);
    const float eta = as_is ? eta_as_is : eta_scaled;
    const float w = fminf(fmaxf(1.5f - eta, 0.f), 1.f);
    return lim + (fr - lim) * w;
  }
}

// Both of a cell's edge increments at once, lim(a, b) toward the upper face and lim(b, a) from the
// lower one. Koren's smoothness measure (far^2 + near^2) / scale^2 and its weight are symmetric in
// the two differences, as the reference computes them in float64: formed once for the pair (a
// single rounding order, where forming it per call let a fused multiply-add round the two orders
// apart), as are the sign test and the twice-the-smaller bound. Other limiters: two calls.
template <int R>
__device__ __forceinline__ void limit_pair(float a, float b, float scale, float& up, float& dn) {
  if constexpr (R != R_KOREN) {
    up = limit<R>(a, b, scale);
    dn = limit<R>(b, a, scale);
  } else {
    const float fu = (a + 2.f * b) * (1.f / 3.f), fd = (b + 2.f * a) * (1.f / 3.f);
    const bool same = same_sign(a, b);
    const float m2 = fminf(2.f * fabsf(a), 2.f * fabsf(b));
    const float lu = same ? copysignf(fminf(m2, fabsf(fu)), b) : 0.f;
    const float ld = same ? copysignf(fminf(m2, fabsf(fd)), a) : 0.f;
    const float s = 0.01f * scale;
    const float s2 = s * s;
    const bool as_is = ((s2 >= 1e-30f) & (s2 < 1e30f)) | (s == 0.f);
    const float eta_as_is = (a * a + b * b) / fmaxf(s2, 1e-30f);
    const float k = 1.f / fabsf(s);
    const float eta_scaled = (a * k) * (a * k) + (b * k) * (b * k);
    const float eta = as_is ? eta_as_is : eta_scaled;
    const float w = fminf(fmaxf(1.5f - eta, 0.f), 1.f);
    up = lu + (fu - lu) * w;
    dn = ld + (fd - ld) * w;
  }
}

// The limiters whose edge increment is the same slope at both faces (lim(a, b) == lim(b, a)).
template <int R>
__host__ __device__ constexpr bool symmetric_limiter() { return R == R_MINMOD || R == R_MC || R == R_VANLEER; }

// hydro.ts:65-83 isenInc and :260-265 isen, for both faces of a cell at once: moves the density
// increments toward the face (up) and from the lower face (dn) toward those along the adiabat,
// by the shared bound at most. m, c, p: (rho, vx, vy, vz, p, s, cs) of the lower neighbour, the
// cell and the upper neighbour; pu, pd: the cell's pressure increments at the two faces.
template <int R, bool PAIR = true>
__device__ __forceinline__ void isen_blend(const float* m, const float* c, const float* p, float pu, float pd,
                                           float inv_gamma, float& up, float& dn) {
  const float rl = m[0], pl = m[4], rc = c[0], pc = c[4], rr = p[0], pr = p[4];
  // (hydro.ts:68: no increment unless all six are positive; the blend below is formed either way
  // and kept only then, a select rather than a branch)
  const bool ok = (rl > 0.f) & (pl > 0.f) & (rc > 0.f) & (pc > 0.f) & (rr > 0.f) & (pr > 0.f);
  const float gi = inv_gamma;
  const float tl = rl * powf(pc / pl, gi) - rc;
  const float tr = rr * powf(pc / pr, gi) - rc;
  const float fade_s = fminf(fmaxf(2.f - fmaxf(fabsf(pl - pc), fabsf(pr - pc)) / (0.2f * pc), 0.f), 1.f);
  const float fade_a = fminf(fmaxf(2.f - fmaxf(fabsf(tl), fabsf(tr)) / (0.01f * rc), 0.f), 1.f);
  const float dvr = sqrtf((p[1] - c[1]) * (p[1] - c[1]) + (p[2] - c[2]) * (p[2] - c[2]) + (p[3] - c[3]) * (p[3] - c[3]));
  const float dvl = sqrtf((c[1] - m[1]) * (c[1] - m[1]) + (c[2] - m[2]) * (c[2] - m[2]) + (c[3] - m[3]) * (c[3] - m[3]));
  const float fade_v = fminf(fmaxf(2.f - fmaxf(dvr, dvl) / (0.1f * fmaxf(c[6], 1e-30f)), 0.f), 1.f);
  const float bound = fmaxf(0.25f * fminf(fabsf(rc - rl), fabsf(rr - rc)), 0.01f * rc * fade_s * fade_a * fade_v);
  float d_up, d_dn;
  if constexpr (PAIR) {
    limit_pair<R>(-tl, tr, rc, d_up, d_dn);
  } else {
    d_up = limit<R>(-tl, tr, rc);
    d_dn = limit<R>(tr, -tl, rc);
  }
  {
    const float d = d_up;
    const float pf = pc + 0.5f * pu;
    const float rf = fminf(fmaxf((rc + 0.5f * d) * powf(fmaxf(pf, 1e-30f) / pc, gi), fminf(rc, rr)), fmaxf(rc, rr));
    const float inc = 2.f * (rf - rc);
    up += ok ? fminf(fmaxf(inc - up, -bound), bound) : 0.f;
  }
  {
    const float d = d_dn;
    const float pf = pc - 0.5f * pd;
    const float rf = fminf(fmaxf((rc - 0.5f * d) * powf(fmaxf(pf, 1e-30f) / pc, gi), fminf(rc, rl)), fmaxf(rc, rl));
    const float inc = -2.f * (rf - rc);
    dn += ok ? fminf(fmaxf(inc - dn, -bound), bound) : 0.f;
  }
}

// Colella & Woodward (1984) parabola edges (their eqs. 1.6, 1.8 and 1.10) from five cells;
// no counterpart in the reference. Returns twice the increments toward the upper face and
// from the lower face, in the reference's edge-increment convention (hydro.ts:282-293).
// The limited slope (eq. 1.8) from the differences toward the cell (dl = a - a_-) and away from
// it (dr = a_+ - a); a cell's two differences are its neighbours' too, so they are formed once.
// The test for an extremum is the product's sign, as the oracle's restatement forms it.
__device__ __forceinline__ float ppm_slope_d(float dl, float dr) {
  const float d = 0.5f * (dl + dr);
  const float m = fminf(fabsf(d), 2.f * fminf(fabsf(dl), fabsf(dr)));
  return (dl * dr > 0.f) ? copysignf(m, d) : 0.f;
}
__device__ __forceinline__ float ppm_slope(float am, float a, float ap) { return ppm_slope_d(a - am, ap - a); }
// The edge increments of one cell from its neighbours and the limited slopes at the cells below,
// at and above it (dm, d0, dp): a sweep that has the slopes already (carried along its march) gives
// them here.
__device__ __forceinline__ void ppm_incs_d(float am, float a, float ap, float dm, float d0, float dp, float& su,
                                           float& sd) {
  const float al = 0.5f * (am + a) - (d0 - dm) * (1.f / 6.f);
  const float ar = 0.5f * (a + ap) - (dp - d0) * (1.f / 6.f);
  // the monotonicity cases by selects (the same values as branches, without divergence): a local
  // extremum flattens the parabola; an overshooting edge is pulled in
  const bool flat = (ar - a) * (a - al) <= 0.f;
  const float da = ar - al, a6 = 6.f * (a - 0.5f * (al + ar));
  const bool pull_l = da * a6 > da * da;
  const bool pull_r = (!pull_l) & (-da * da > da * a6);
  const float al2 = flat ? a : (pull_l ? 3.f * a - 2.f * ar : al);
  const float ar2 = flat ? a : (pull_r ? 3.f * a - 2.f * al : ar);
  su = 2.f * (ar2 - a);
  sd = 2.f * (a - al2);
}
__device__ __forceinline__ void ppm_incs(float a2m, float am, float a, float ap, float a2p, float& su, float& sd) {
  const float d1 = am - a2m, d2 = a - am, d3 = ap - a, d4 = a2p - ap;
  ppm_incs_d(am, a, ap, ppm_slope_d(d1, d2), ppm_slope_d(d2, d3), ppm_slope_d(d3, d4), su, sd);
}

// The edge increments of one cell along one axis (hydro.ts:282-293; the ghost form :347-356):
// su toward the upper face, sd from the lower face, for (rho, vx, vy, vz, p, s).
// m2, p2 (two cells away) are read by PPM only. PAIR (Koren): a cell's two increments formed as a
// pair (limit_pair) rather than by two calls; the 2D row march keeps two calls, which its register
// budget schedules better.
template <int R, bool ISEN, bool PAIR = true>
__device__ __forceinline__ void axis_edges(const float* m2, const float* m, const float* c, const float* p, const float* p2,
                                           float inv_gamma, float* su, float* sd) {
  if constexpr (R == R_PPM) {
#pragma unroll
    for (int v = 0; v < 6; v++) ppm_incs(m2[v], m[v], c[v], p[v], p2[v], su[v], sd[v]);
  } else {
    // hydro.ts:268-270 scales: density, sound speed for velocities, pressure, none for s.
    const float sc[6] = {c[0], c[6], c[6], c[6], c[4], 0.f};
#pragma unroll
    for (int v = 0; v < 6; v++) {
      if constexpr (symmetric_limiter<R>()) {
        su[v] = limit<R>(c[v] - m[v], p[v] - c[v], sc[v]);
        sd[v] = su[v];
      } else if constexpr (PAIR) {
        limit_pair<R>(c[v] - m[v], p[v] - c[v], sc[v], su[v], sd[v]);
      } else {
        su[v] = limit<R>(c[v] - m[v], p[v] - c[v], sc[v]);
        sd[v] = limit<R>(p[v] - c[v], c[v] - m[v], sc[v]);
      }
    }
    if constexpr (ISEN) isen_blend<R, PAIR>(m, c, p, su[4], sd[4], inv_gamma, su[0], sd[0]);
  }
}

// hydro.ts:360-375 side, rotated so that index 1 is normal to the face; then
// hydro.ts:102-159 riemannFlux. L and R are (rho, vx, vy, vz, p, s, shock flag). The flux comes
// back in the lab frame: (m, mx, my, mz, e, ei, s, vn).
// The three regions (left-supersonic, right-supersonic, star) and the star side are chosen by
// selects rather than branches, so that a warp whose faces fall in different regions runs one
// path; the values computed for the regions not chosen are discarded.
// hll_any: false when the caller knows that neither side of any face it solves is shock-flagged
// (a CTA-uniform fact, so the branch does not diverge). The HLL flux then has weight 0 and is
// skipped; a face of weight 0 takes the HLLC flux as it is either way.
template <int AXIS>
__device__ __forceinline__ void riemann(const float* L, const float* R, const KParams& P, float* F,
                                        bool hll_any = true) {
  constexpr int A0 = 1 + AXIS, A1 = 1 + (AXIS + 1) % 3, A2 = 1 + (AXIS + 2) % 3;
  const float lr = fmaxf(L[0], P.rho_floor), rr = fmaxf(R[0], P.rho_floor);
  const float lp = fmaxf(L[4], P.p_floor), rp = fmaxf(R[4], P.p_floor);
  const float lu = L[A0], lv = L[A1], lw = L[A2];
  const float ru = R[A0], rv = R[A1], rw = R[A2];
  const float lc = sqrtf(P.gamma * lp / lr), rc = sqrtf(P.gamma * rp / rr);
  const float lei = lp * P.inv_gm1, rei = rp * P.inv_gm1;
  const float w_hll = P.hll ? 1.f : fmaxf(L[6], R[6]);

  const float sl = fminf(lu - lc, ru - rc);
  const float sr = fmaxf(lu + lc, ru + rc);
  const float el = lei + 0.5f * lr * (lu * lu + lv * lv + lw * lw);
  const float er = rei + 0.5f * rr * (ru * ru + rv * rv + rw * rw);
  const float ml0 = lr * lu, ml1 = lr * lv, ml2 = lr * lw;
  const float mr0 = rr * ru, mr1 = rr * rv, mr2 = rr * rw;
  const float fpl0 = ml0 * lu + lp, fpl1 = ml1 * lu, fpl2 = ml2 * lu;
  const float fpr0 = mr0 * ru + rp, fpr1 = mr1 * ru, fpr2 = mr2 * ru;
  const float fel = (el + lp) * lu, fer = (er + rp) * ru;

  // HLL state flux and the contact speed
  const float ql = lr * (sl - lu);
  const float qr = rr * (sr - ru);
  const float sm = (rp - lp + lu * ql - ru * qr) / (ql - qr);
  // HLLC star state on the side of the contact the face lies on
  const bool left = sm >= 0.f;
  const float sK = left ? sl : sr, qK = left ? ql : qr, rK = left ? lr : rr, uK = left ? lu : ru;
  const float vK = left ? lv : rv, wK = left ? lw : rw, pK = left ? lp : rp, eK = left ? el : er;
  const float mK0 = left ? ml0 : mr0, mK1 = left ? ml1 : mr1, mK2 = left ? ml2 : mr2;
  const float fK0 = left ? fpl0 : fpr0, fK1 = left ? fpl1 : fpr1, fK2 = left ? fpl2 : fpr2, feK = left ? fel : fer;
  const float f = qK / (sK - sm);
  const float es = f * (eK / rK + (sm - uK) * (sm + pK / qK));
  const float cm = mK0 + sK * (f - rK);
  const float c0 = fK0 + sK * (f * sm - mK0);
  const float c1 = fK1 + sK * (f * vK - mK1);
  const float c2 = fK2 + sK * (f * wK - mK2);
  const float ce = feK + sK * (es - eK);
  float m = cm, p0 = c0, p1 = c1, p2 = c2, e = ce;
  if (hll_any || P.hll) {
    const float inv = 1.f / (sr - sl);
    const float slsr = sl * sr;
    const float hm = (sr * ml0 - sl * mr0 + slsr * (rr - lr)) * inv;
    const float hp0 = (sr * fpl0 - sl * fpr0 + slsr * (mr0 - ml0)) * inv;
    const float hp1 = (sr * fpl1 - sl * fpr1 + slsr * (mr1 - ml1)) * inv;
    const float hp2 = (sr * fpl2 - sl * fpr2 + slsr * (mr2 - ml2)) * inv;
    const float he = (sr * fel - sl * fer + slsr * (er - el)) * inv;
    // a face of weight 0 keeps the HLLC flux exactly, as where the HLL one was skipped: the
    // result does not depend on which faces share a CTA (c + (h - c) * 0 can turn -0 into +0)
    const bool blend = w_hll != 0.f;
    m = blend ? cm + (hm - cm) * w_hll : cm;
    p0 = blend ? c0 + (hp0 - c0) * w_hll : c0;
    p1 = blend ? c1 + (hp1 - c1) * w_hll : c1;
    p2 = blend ? c2 + (hp2 - c2) * w_hll : c2;
    e = blend ? ce + (he - ce) * w_hll : ce;
  }
  float vn = sm;
  // supersonic faces take the upwind side's flux
  const bool supl = sl >= 0.f, supr = sr <= 0.f;
  m = supl ? ml0 : (supr ? mr0 : m);
  p0 = supl ? fpl0 : (supr ? fpr0 : p0);
  p1 = supl ? fpl1 : (supr ? fpr1 : p1);
  p2 = supl ? fpl2 : (supr ? fpr2 : p2);
  e = supl ? fel : (supr ? fer : e);
  vn = supl ? lu : (supr ? ru : vn);
  const bool up = m >= 0.f;
  F[0] = m;
  F[A0] = p0;
  F[A1] = p1;
  F[A2] = p2;
  F[4] = e;
  F[5] = m * ((up ? lei : rei) / (up ? lr : rr));
  F[6] = m * (up ? L[5] : R[5]);
  F[7] = vn;
}

// Primitives of one cell from its conserved state (hydro.ts:233-257 primitives; prim.wgsl:26-51):
// (rho, vx, vy, vz, p, s, cs), velocities multiplied by the boundary signs f.
__device__ __forceinline__ void prim_from_cons(const float4 a, const float4 b, const KParams& P, float fx, float fy,
                                               float fz, float* w) {
  const float rho = fmaxf(a.x, P.rho_floor);
  const float inv = 1.f / rho;
  float p = P.gm1 * b.y;
  if (!(p >= P.p_floor)) p = P.p_floor;
  w[0] = rho;
  w[1] = a.y * inv * fx;
  w[2] = a.z * inv * fy;
  w[3] = a.w * inv * fz;
  w[4] = p;
  w[5] = b.z * inv;
  w[6] = sqrtf(P.gamma * p * inv);
}

// The six primitives the stencil reads of a neighbour (rho, vx, vy, vz, p, s): the sound
// speed is needed only at the centre cell and is formed there (with_cs).
__device__ __forceinline__ void prim6_from_cons(const float4 a, const float4 b, const KParams& P, float fx, float fy,
                                                float fz, float* w) {
  const float rho = fmaxf(a.x, P.rho_floor);
  const float inv = 1.f / rho;
  float p = P.gm1 * b.y;
  if (!(p >= P.p_floor)) p = P.p_floor;
  w[0] = rho;
  w[1] = a.y * inv * fx;
  w[2] = a.z * inv * fy;
  w[3] = a.w * inv * fz;
  w[4] = p;
  w[5] = b.z * inv;
}
__device__ __forceinline__ void with_cs(float* w, const KParams& P) { w[6] = sqrtf(P.gamma * w[4] / w[0]); }

// The signal rate of a cell (hydro.ts:254): |vx| + |vy| + |vz| + signal * cs.
__device__ __forceinline__ float signal_rate(const float4 a, const float4 b, const KParams& P) {
  float w[7];
  prim_from_cons(a, b, P, 1.f, 1.f, 1.f, w);
  return fabsf(w[1]) + fabsf(w[2]) + fabsf(w[3]) + P.signal * w[6];
}

// hydro.ts:216-220 bcAxis: the source index of a possibly out-of-range index and the sign of
// the velocity along that axis. Indices beyond the reach of the scheme are clamped into range
// (they feed no output).
// Boundary codes: 0 periodic, 1 outflow, 2 reflect (the reference's), and 3 halo: a z face of one
// slab of a larger grid, whose ghost planes are stored beyond the slab and filled by the caller
// with the neighbouring slab's planes.
constexpr int BC_HALO = 3;
// Whether a face's ghosts take the adjacent inner cell's half step (outflow and reflect).
__host__ __device__ __forceinline__ bool bc_inner(int code) { return code == 1 || code == 2; }

__device__ __forceinline__ int bc_map(int i, int n, int lo, int hi, float& f) {
  f = 1.f;
  if (i < 0) {
    if (lo == 0) i = ((i % n) + n) % n;
    else if (lo == 1) i = 0;
    else { i = -1 - i; f = -1.f; }
  } else if (i >= n) {
    if (hi == 0) i = i % n;
    else if (hi == 1) i = n - 1;
    else { i = 2 * n - 1 - i; f = -1.f; }
  }
  return min(max(i, 0), n - 1);
}

}  // namespace shz
