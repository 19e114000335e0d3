// Per-cell steps of the hydro scheme shared by the uniform sweep (sweep.cu) and the block passes
// of the adaptive grid (amr_kernels.cu): the Hancock predictor, face states and the update.
#pragma once
#include "hydro_math.cuh"

namespace shz {

// The per-cell result of the predictor (hydro.ts:272-322 predictRaw): the half-step state q,
// the shock flag and the first-order flag.
struct Pred {
  float q[6];
  float flag;
  bool fo;
};

// The shock detector's pressure jump along one axis (hydro.ts:300-303: |p+ - p-| / min(p+, p-)
// above the threshold), as its excess over the threshold: |p+ - p-| - threshold min(p+, p-), which
// is positive exactly where the ratio exceeds it (the pressures are floored, so positive), without
// the division. The largest over the axes decides.
__device__ __forceinline__ float jump_excess(float pm, float pp, float thresh) {
  return fabsf(pp - pm) - thresh * fminf(pp, pm);
}

// hydro.ts:294-321: slopes -> shock flag -> Hancock half step -> positivity fallback, given the
// edge increments su/sd per active axis, the convergence, and the largest jump_excess over the axes.
template <int DIM>
__device__ __forceinline__ void hancock(const float* c, float conv, float jump, const float (*su)[6], const float (*sd)[6],
                                        float h, const KParams& P, Pred& out) {
  float big = 0.f, fall = 0.f, dv = 0.f;
  float adv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float gradp[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int a = 0; a < DIM; a++) {
    big = fmaxf(big, fmaxf(fabsf(su[a][4]), fabsf(sd[a][4])));
    fall = fminf(fall, fminf(0.5f * su[a][0], -0.5f * sd[a][0]));
    const float va = c[1 + a];
#pragma unroll
    for (int v = 0; v < 6; v++) adv[v] += va * (0.5f * (su[a][v] + sd[a][v]));
    dv += 0.5f * (su[a][1 + a] + sd[a][1 + a]);
    gradp[a] = 0.5f * (su[a][4] + sd[a][4]);
  }
  out.flag = ((conv < 0.f) & (jump > 0.f)) ? 1.f : 0.f;
  const float rho = c[0], cs = c[6];
  const float inv_rho = 1.f / rho;
  float qh[6];
  qh[0] = rho - h * (adv[0] + rho * dv);
#pragma unroll
  for (int d = 0; d < 3; d++) qh[1 + d] = c[1 + d] - h * (adv[1 + d] + gradp[d] * inv_rho);
  qh[4] = c[4] - h * (adv[4] + rho * cs * cs * dv);
  qh[5] = c[5] - h * adv[5];
  const float rmin = qh[0] + fall;
  const float pmin = qh[4] - 0.5f * big;
  out.fo = !((rmin > 0.f) & (pmin > 0.f));
#pragma unroll
  for (int v = 0; v < 6; v++) out.q[v] = out.fo ? c[v] : qh[v];
}

// Face state q + 0.5 sgn inc (q alone when first order: the increments are zeroed), with the
// cell's shock flag (hydro.ts:362 side's f(n)).
__device__ __forceinline__ void face_state(const Pred& pr, const float* inc, float sgn, float* f) {
  const float k = pr.fo ? 0.f : 0.5f * sgn;
#pragma unroll
  for (int v = 0; v < 6; v++) f[v] = pr.q[v] + k * inc[v];
  f[6] = pr.flag;
}

// The update of one cell (hydro.ts:422-446): conservative update, dual-energy switch and floors.
// acc = (dm, dmx, dmy, dmz, de, dei, ds, dvn) summed with the reference's signs; ph = the
// cell's half-step pressure.
__device__ __forceinline__ void update_cell(const float4 a, const float4 b, const float* acc, float ph, float dtdx,
                                            const KParams& P, float4& na, float4& nb) {
  const float rho = fmaxf(a.x + dtdx * acc[0], P.rho_floor);
  const float mx = a.y + dtdx * acc[1], my = a.z + dtdx * acc[2], mz = a.w + dtdx * acc[3];
  float E = b.x + dtdx * acc[4];
  float eint = b.y + dtdx * (acc[5] + fmaxf(ph, P.p_floor) * acc[7]);
  const float ke = (0.5f * (mx * mx + my * my + mz * mz)) / rho;
  const float eth = E - ke;
  const float emin = P.e_floor;
  // the dual-energy switch by selects (a warp whose cells choose differently runs one path)
  const bool from_total = (eth > P.eta_dual * E) & (eth >= emin);
  const float eadv = (eint >= emin) ? eint : emin;
  eint = from_total ? eth : eadv;
  E = from_total ? E : ke + eadv;
  na = make_float4(rho, mx, my, mz);
  nb = make_float4(E, eint, b.z + dtdx * acc[6], b.w);
}

}  // namespace shz

namespace shz {

// The Hancock step with the half-step slopes of some axes masked out (hydro/predictor.wgsl
// `mask`): a ghost next to a coarser block at the rim of its face has no transverse neighbours,
// so its slopes along those axes do not drive the half step. The positivity check still sees
// every increment, as in the reference.
template <int DIM>
__device__ __forceinline__ void hancock_masked(const float* c, float conv, float jump, const float (*su)[6],
                                               const float (*sd)[6], const float* mask, float h, const KParams& P,
                                               Pred& out) {
  float big = 0.f, fall = 0.f, dv = 0.f;
  float adv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float gradp[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int a = 0; a < DIM; a++) {
    big = fmaxf(big, fmaxf(fabsf(su[a][4]), fabsf(sd[a][4])));
    fall = fminf(fall, fminf(0.5f * su[a][0], -0.5f * sd[a][0]));
    const float va = c[1 + a];
    const float k = 0.5f * mask[a];
#pragma unroll
    for (int v = 0; v < 6; v++) adv[v] += va * (k * (su[a][v] + sd[a][v]));
    dv += k * (su[a][1 + a] + sd[a][1 + a]);
    gradp[a] = k * (su[a][4] + sd[a][4]);
  }
  out.flag = ((conv < 0.f) & (jump > 0.f)) ? 1.f : 0.f;
  const float rho = c[0], cs = c[6];
  const float inv_rho = 1.f / rho;
  float qh[6];
  qh[0] = rho - h * (adv[0] + rho * dv);
#pragma unroll
  for (int d = 0; d < 3; d++) qh[1 + d] = c[1 + d] - h * (adv[1 + d] + gradp[d] * inv_rho);
  qh[4] = c[4] - h * (adv[4] + rho * cs * cs * dv);
  qh[5] = c[5] - h * adv[5];
  const float rmin = qh[0] + fall;
  const float pmin = qh[4] - 0.5f * big;
  out.fo = !((rmin > 0.f) & (pmin > 0.f));
#pragma unroll
  for (int v = 0; v < 6; v++) out.q[v] = out.fo ? c[v] : qh[v];
}

}  // namespace shz
