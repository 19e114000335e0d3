// The reference's two passes in place of the fused sweep (two_pass): amr_predict writes the half
// steps of every leaf and its first ghost layer to their atlas, amr_update reads them for the
// fluxes and the update (amr/predict.wgsl:184-221, amr/update.wgsl:207-560). Kept as the
// cross-check of the fused sweep, and the passes of per-block timesteps (a bin table `bins`, null
// for one timestep): the half-step atlas of a block stays as its step began until its next start,
// which is what its faster neighbours read of it meanwhile.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <type_traits>

#include "amr_device.cuh"

namespace shz {
namespace amrk {

// 2. Half steps of every leaf over its cells and first ghost layer (predict.wgsl:184-221): a
// same-level or boundary ghost is predicted at its source and mirrored; a ghost beside a coarser
// block, or beside a neighbour part way through a longer step (whose ghost the assemble filled
// from its half step), in place, its transverse slopes dropped at the rim of the face. Every
// block predicts with its own step, its ghosts included.
template <int DIM, int R, bool ISEN>
__global__ void __launch_bounds__(NT) amr_predict(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                  const int* __restrict__ list, int n, const float4* __restrict__ w1,
                                                  const float4* __restrict__ w2, float4* __restrict__ p1,
                                                  float4* __restrict__ p2, const DevClock* __restrict__ clks,
                                                  const int* __restrict__ bins) {
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int slot = __ldg(list + i);
    const int g = bt_at(bt, slot, GRID_WORD);
    const KParams& P = gp[g];
    const double dt = clks[g].dt * ldexp(1.0, blk_bin(bins, slot));
    const float h = (float)((0.5 * dt) * ldexp(1.0, bt_at(bt, slot, 0)) / P.dx);
    for (int t = threadIdx.x; t < BG<DIM>::PN; t += NT) {
      int l[3] = {t % PP - 1, (t / PP) % PP - 1, DIM == 3 ? t / (PP * PP) - 1 : 0};
      const Src s = ghost_src<DIM>(bt, slot, l);
      if (s.kind == 2) continue;
      const bool stale = s.kind == 0 && s.slot != slot && mid_block(bt, bins, s.slot);
      const bool at_source = s.kind == 0 && !stale;
      const int src = at_source ? s.slot : slot;
      int c0[3] = {at_source ? s.l[0] : l[0], at_source ? s.l[1] : l[1], at_source ? s.l[2] : l[2]};
      float mask[3] = {1.f, 1.f, 1.f};
      if (!at_source)
#pragma unroll
        for (int a = 0; a < DIM; a++) mask[a] = (l[a] == 0 || l[a] == BS - 1) ? 0.f : 1.f;
      float c[7];
      load_w<DIM>(w1, w2, src, c0, c);
      float su[DIM][6], sd[DIM][6];
      float conv = 0.f, jump = -INFINITY;
#pragma unroll
      for (int a = 0; a < DIM; a++) {
        float m[7], p[7];
        int lm[3] = {c0[0], c0[1], c0[2]}, lp[3] = {c0[0], c0[1], c0[2]};
        lm[a] -= 1;
        lp[a] += 1;
        load_w<DIM>(w1, w2, src, lm, m);
        load_w<DIM>(w1, w2, src, lp, p);
        axis_edges<R, ISEN>(m, m, c, p, p, P.inv_gamma, su[a], sd[a]);
        conv += p[1 + a] - m[1 + a];
        jump = fmaxf(jump, jump_excess(m[4], p[4], P.shock_thresh));
      }
      Pred pr;
      hancock_masked<DIM>(c, conv, jump, su, sd, mask, h, P, pr);
      if (at_source) {
        pr.q[1] *= s.flip[0];
        pr.q[2] *= s.flip[1];
        pr.q[3] *= s.flip[2];
      }
      const size_t o = (size_t)slot * BG<DIM>::PN + t;
      p1[o] = make_float4(pr.q[0], pr.q[1], pr.q[2], pr.q[3]);
      p2[o] = make_float4(pr.q[4], pr.q[5], pr.flag, pr.fo ? 1.f : 0.f);
    }
  }
}

// The flux through the face between cells a and a + e_AXIS of block `slot`
// (flux.wgsl flux_between): face states from the half steps and the edge increments the
// primitives give along the axis.
template <int DIM, int R, bool ISEN, int AXIS>
__device__ __forceinline__ void face_flux(const KParams& P, const float4* __restrict__ w1, const float4* __restrict__ w2,
                                          const float4* __restrict__ p1, const float4* __restrict__ p2, int slot,
                                          const int* a, float* F) {
  int am[3] = {a[0], a[1], a[2]}, b[3] = {a[0], a[1], a[2]}, bp[3] = {a[0], a[1], a[2]};
  am[AXIS] -= 1;
  b[AXIS] += 1;
  bp[AXIS] += 2;
  float wm[7], wa[7], wb[7], wbp[7];
  load_w<DIM>(w1, w2, slot, am, wm);
  load_w<DIM>(w1, w2, slot, a, wa);
  load_w<DIM>(w1, w2, slot, b, wb);
  load_w<DIM>(w1, w2, slot, bp, wbp);
  float su[6], sd[6], tu[6], td[6];
  axis_edges<R, ISEN>(wm, wm, wa, wb, wb, P.inv_gamma, su, sd);   // cell a: toward its upper face
  axis_edges<R, ISEN>(wa, wa, wb, wbp, wbp, P.inv_gamma, tu, td);  // cell b: from its lower face
  Pred pa, pb;
  {
    const size_t o = (size_t)slot * BG<DIM>::PN + ptex<DIM>(a);
    const float4 x = __ldg(p1 + o), y = __ldg(p2 + o);
    pa.q[0] = x.x; pa.q[1] = x.y; pa.q[2] = x.z; pa.q[3] = x.w; pa.q[4] = y.x; pa.q[5] = y.y;
    pa.flag = y.z;
    pa.fo = y.w != 0.f;
  }
  {
    const size_t o = (size_t)slot * BG<DIM>::PN + ptex<DIM>(b);
    const float4 x = __ldg(p1 + o), y = __ldg(p2 + o);
    pb.q[0] = x.x; pb.q[1] = x.y; pb.q[2] = x.z; pb.q[3] = x.w; pb.q[4] = y.x; pb.q[5] = y.y;
    pb.flag = y.z;
    pb.fo = y.w != 0.f;
  }
  float L[7], Rr[7];
  face_state(pa, su, 1.f, L);
  face_state(pb, td, -1.f, Rr);
  riemann<AXIS>(L, Rr, P, F);
}

// The fine-flux matching of a face at the edge of a block (amr/update.wgsl:207-295): where the
// same-level neighbour beyond it is refined, the face's flux is the mean of the fluxes through
// the 2^(ndim-1) fine faces it covers, computed as the fine leaf computes them. With per-block
// timesteps (kb: this block's bin; deposit: it is half way through its step) each neighbour's
// flux counts for its share of this block's step (update.wgsl:182-186): half for a faster
// neighbour, all of it for one in step, none in a deposit; and a same-level leaf that steps
// twice as often gives its own flux through the face for half of the step. Returns whether the
// face took a neighbour's flux.
__device__ __forceinline__ float bin_share(const int* __restrict__ bins, int nb, int kb, bool deposit) {
  if (!bins) return 1.f;
  if (blk_bin(bins, nb) < kb) return 0.5f;
  return deposit ? 0.f : 1.f;
}
template <int DIM, int R, bool ISEN, int AXIS>
__device__ __forceinline__ bool match_face(const KParams& P, const int* __restrict__ bt, const float4* __restrict__ w1,
                                           const float4* __restrict__ w2, const float4* __restrict__ p1,
                                           const float4* __restrict__ p2, int slot, const int* l, bool hi, float* F,
                                           const int* __restrict__ bins = nullptr, int kb = 0, bool deposit = false) {
  const int np = bt_at(bt, slot, 6 + 2 * AXIS + (hi ? 1 : 0));
  if (np < 0) return false;
  const bool upper = !hi;
  if (leaf_of(bt, np)) {
    // a same-level leaf in a faster bin: its flux through the face, from its own half steps
    if (!bins || np == slot || blk_bin(bins, np) >= kb) return false;
    int a[3] = {l[0], l[1], l[2]};
    a[AXIS] = upper ? BS - 1 : -1;
    float f[8];
    face_flux<DIM, R, ISEN, AXIS>(P, w1, w2, p1, p2, np, a, f);
#pragma unroll
    for (int v = 0; v < 8; v++) F[v] = f[v] * 0.5f;
    return true;
  }
  int h[3] = {l[0] >= BS / 2, l[1] >= BS / 2, DIM == 3 ? (l[2] >= BS / 2) : 0};
  int bits[3] = {h[0], h[1], h[2]};
  bits[AXIS] = upper ? 1 : 0;
  if (DIM == 2) bits[2] = 0;
  const int ch = bt_at(bt, np, 12 + (bits[0] | (bits[1] << 1) | (bits[2] << 2)));
  if (ch < 0) return false;
  const float part = bin_share(bins, ch, kb, deposit);
  if (part == 0.f) {
#pragma unroll
    for (int v = 0; v < 8; v++) F[v] = 0.f;
    return false;
  }
  int a0[3] = {2 * (l[0] - (BS / 2) * h[0]), 2 * (l[1] - (BS / 2) * h[1]), DIM == 3 ? 2 * (l[2] - (BS / 2) * h[2]) : 0};
  a0[AXIS] = upper ? BS - 1 : -1;
  constexpr int T1 = (AXIS + 1) % 3, T2 = (AXIS + 2) % 3;
  const int n1 = (DIM == 2 && T1 == 2) ? 1 : 2;
  const int n2 = (DIM == 2 && T2 == 2) ? 1 : 2;
  float sum[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int j = 0; j < n2; j++)
    for (int i = 0; i < n1; i++) {
      int a[3] = {a0[0], a0[1], a0[2]};
      a[T1] += i;
      a[T2] += j;
      float f[8];
      face_flux<DIM, R, ISEN, AXIS>(P, w1, w2, p1, p2, ch, a, f);
#pragma unroll
      for (int v = 0; v < 8; v++) sum[v] += f[v];
    }
  float w = 1.f / (float)(n1 * n2);
  if (bins) w *= part;
#pragma unroll
  for (int v = 0; v < 8; v++) F[v] = sum[v] * w;
  return true;
}

// 3. Fluxes and the update of every leaf (update.wgsl:327-560). A CTA takes a block plane by
// plane along z; each thread owns a column and solves its lower x and y faces (the last row
// also the block's upper face) into shared memory, and its z faces in registers, so every face
// is solved once.
// With per-block timesteps each block steps with its own dt, and a leaf half way through its step
// that has a faster neighbour takes a deposit (update.wgsl:339-445): no fluxes of its own, only
// its faster neighbours' second-step fluxes through the shared faces, with the half-step pressure
// of its step's start; a cell on no such face keeps its state. The state is then updated in place
// (o1, o2 the same arrays as u1, u2): a cell is read and written by one thread only, and every
// neighbour the pass reads is in the primitive and half-step atlases.
template <int DIM, int R, bool ISEN>
__global__ void __launch_bounds__(NT) amr_update(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                 const int* __restrict__ list, int n, const float4* u1,
                                                 const float4* u2, const float4* __restrict__ w1,
                                                 const float4* __restrict__ w2, const float4* __restrict__ p1,
                                                 const float4* __restrict__ p2, float4* o1,
                                                 float4* o2, const DevClock* __restrict__ clks,
                                                 const int* __restrict__ bins) {
  __shared__ float sFx[8][BS * (BS + 1)];
  __shared__ float sFy[8][BS * (BS + 1)];
  const int tx = threadIdx.x % BS, ty = threadIdx.x / BS;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int slot = __ldg(list + i);
    const int g = bt_at(bt, slot, GRID_WORD);
    const KParams& P = gp[g];
    const int kb = blk_bin(bins, slot);
    const bool dep = bins != nullptr && !blk_active(bins, slot);
    const double dt = clks[g].dt * ldexp(1.0, kb);
    const bool held = clks[g].held != 0;
    const float dtdx = (float)(dt * ldexp(1.0, bt_at(bt, slot, 0)) / P.dx);
    float Fzlo[8];
    const int nk = DIM == 3 ? BS : 1;
    // this block's own flux through the face above cell a along AXIS (none in a deposit)
    auto own = [&](auto axis_tag, const int* a, float* F) {
      constexpr int AX = decltype(axis_tag)::value;
      if (dep) {
#pragma unroll
        for (int v = 0; v < 8; v++) F[v] = 0.f;
      } else {
        face_flux<DIM, R, ISEN, AX>(P, w1, w2, p1, p2, slot, a, F);
      }
    };
    using X0 = std::integral_constant<int, 0>;
    using X1 = std::integral_constant<int, 1>;
    using X2 = std::integral_constant<int, 2>;
    for (int k = 0; k < nk; k++) {
      int l[3] = {tx, ty, k};
      float F[8];
      bool touched = false;  // a face of this cell took a faster neighbour's flux
      // x faces
      {
        int a[3] = {tx - 1, ty, k};
        own(X0{}, a, F);
        if (tx == 0) touched |= match_face<DIM, R, ISEN, 0>(P, bt, w1, w2, p1, p2, slot, l, false, F, bins, kb, dep);
#pragma unroll
        for (int v = 0; v < 8; v++) sFx[v][ty * (BS + 1) + tx] = F[v];
        if (tx == BS - 1) {
          own(X0{}, l, F);
          touched |= match_face<DIM, R, ISEN, 0>(P, bt, w1, w2, p1, p2, slot, l, true, F, bins, kb, dep);
#pragma unroll
          for (int v = 0; v < 8; v++) sFx[v][ty * (BS + 1) + BS] = F[v];
        }
      }
      // y faces
      {
        int a[3] = {tx, ty - 1, k};
        own(X1{}, a, F);
        if (ty == 0) touched |= match_face<DIM, R, ISEN, 1>(P, bt, w1, w2, p1, p2, slot, l, false, F, bins, kb, dep);
#pragma unroll
        for (int v = 0; v < 8; v++) sFy[v][ty * BS + tx] = F[v];
        if (ty == BS - 1) {
          own(X1{}, l, F);
          touched |= match_face<DIM, R, ISEN, 1>(P, bt, w1, w2, p1, p2, slot, l, true, F, bins, kb, dep);
#pragma unroll
          for (int v = 0; v < 8; v++) sFy[v][BS * BS + tx] = F[v];
        }
      }
      float Fzhi[8];
      if constexpr (DIM == 3) {
        if (k == 0) {
          int a[3] = {tx, ty, -1};
          own(X2{}, a, Fzlo);
          touched |= match_face<DIM, R, ISEN, 2>(P, bt, w1, w2, p1, p2, slot, l, false, Fzlo, bins, kb, dep);
        }
        own(X2{}, l, Fzhi);
        if (k == BS - 1) touched |= match_face<DIM, R, ISEN, 2>(P, bt, w1, w2, p1, p2, slot, l, true, Fzhi, bins, kb, dep);
      }
      __syncthreads();
      float acc[8];
#pragma unroll
      for (int v = 0; v < 8; v++) {
        float x = sFx[v][ty * (BS + 1) + tx];
        x -= sFx[v][ty * (BS + 1) + tx + 1];
        x += sFy[v][ty * BS + tx];
        x -= sFy[v][(ty + 1) * BS + tx];
        if constexpr (DIM == 3) {
          x += Fzlo[v];
          x -= Fzhi[v];
        }
        acc[v] = x;
      }
      const size_t oc = (size_t)slot * BG<DIM>::CB + cell_ix<DIM>(l);
      const size_t op = (size_t)slot * BG<DIM>::PN + ptex<DIM>(l);
      const float4 a = u1[oc], b = u2[oc];
      if (held || (dep && !touched)) {
        o1[oc] = a;
        o2[oc] = b;
      } else {
        float4 na, nb;
        update_cell(a, b, acc, __ldg(p2 + op).x, dtdx, P, na, nb);
        o1[oc] = na;
        o2[oc] = nb;
      }
      if constexpr (DIM == 3) {
#pragma unroll
        for (int v = 0; v < 8; v++) Fzlo[v] = Fzhi[v];
      }
      __syncthreads();
    }
  }
}

}  // namespace amrk

// Host launchers.

cudaError_t amr_launch_predict(const AmrLaunch& L, const int* list, int n, const DevClock* clks, cudaStream_t s,
                               const int* bins) {
  if (n <= 0) return cudaSuccess;
  const int g = grid_for(n, 4);
  if (L.ndim == 3) {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_predict<3, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, L.w1, L.w2, L.p1, L.p2, clks, bins))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_predict<3, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, L.w1, L.w2, L.p1, L.p2, clks, bins))) }
  } else {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_predict<2, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, L.w1, L.w2, L.p1, L.p2, clks, bins))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_predict<2, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, L.w1, L.w2, L.p1, L.p2, clks, bins))) }
  }
  return cudaGetLastError();
}

cudaError_t amr_launch_update(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, float4* o1,
                              float4* o2, const DevClock* clks, cudaStream_t s, const int* bins) {
  if (n <= 0) return cudaSuccess;
  const int g = grid_for(n, 4);
  if (L.ndim == 3) {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_update<3, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, L.p1, L.p2, o1, o2, clks, bins))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_update<3, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, L.p1, L.p2, o1, o2, clks, bins))) }
  } else {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_update<2, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, L.p1, L.p2, o1, o2, clks, bins))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_update<2, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, L.p1, L.p2, o1, o2, clks, bins))) }
  }
  return cudaGetLastError();
}

}  // namespace shz
