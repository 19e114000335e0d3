// The fused block sweep of the adaptive grid and the fine-flux pre-pass it reads.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <functional>
#include <vector>

#include "amr_device.cuh"
#include "tma.cuh"

namespace shz {
namespace amrk {

// The fused block sweep: predict, fluxes and update of a leaf in one pass over its primitive
// atlas (which assemble filled, ghosts and edges included), so that each edge increment is formed
// once and no half-step atlas is written. A CTA takes a block as the uniform sweep (sweep.cu)
// takes a column: its (16 + 2)^2 threads march the 16 planes along z; the primitives of three
// planes sit in shared memory.
//
// Ghosts, by the block-table entry of their face:
//   same level (a slot): predicted in place: the atlas holds the neighbour's cells and, across
//     edges, what the neighbour's own ghosts hold, so this is the prediction at the source
//     (amr/predict.wgsl:196-206);
//   one level coarser (NB_COARSE): predicted in place, the slopes along the face's transverse
//     axes dropped at the rim of the face (amr/predict.wgsl:207-214);
//   a domain boundary: the half-step state of the cell it maps to, mirrored for a wall, with edge
//     increments at the ghost position (hydro.ts:329-358, as amr/predict.wgsl's at-source rule).
// A face whose same-level neighbour is refined takes the mean of the fine fluxes through it
// (amr/update.wgsl:207-295), the fine cells predicted from the fine leaf's atlas by predict_texel.

constexpr int SX = BS + 2;        // threads per row: the block and one ghost on each side
constexpr int SNT = SX * SX;      // 324 threads
constexpr int SPN = SX * SX;      // predictor region per plane
constexpr int SWN = PAD * PAD;    // primitive texels per plane


// The seven primitives of texel l of a block's atlas (the sound speed as the atlas holds it).
template <int DIM>
__device__ __forceinline__ void load_w7(const float4* __restrict__ w1, const float4* __restrict__ w2, int slot, const int* l,
                                        float* w) {
  const size_t o = (size_t)slot * BG<DIM>::WN + wtex<DIM>(l);
  const float4 a = __ldg(w1 + o), b = __ldg(w2 + o);
  w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
  w[4] = b.x; w[5] = b.y; w[6] = b.z;
}

template <int DIM>
__device__ __forceinline__ void load_w6(const float4* __restrict__ w1, const float4* __restrict__ w2, int slot, const int* l,
                                        float* w) {
  const size_t o = (size_t)slot * BG<DIM>::WN + wtex<DIM>(l);
  const float4 a = __ldg(w1 + o), b = __ldg(w2 + o);
  w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
  w[4] = b.x; w[5] = b.y;
}

// The predictor of texel l0 of block `slot`, read from its primitive atlas, under the ghost rules
// above; with the edge increments along `axis` at l0 itself (for its face states on that axis).
// (bins: the per-block timesteps' bin table, or null; a ghost beside a neighbour part way through
// its step is predicted in place, as beside a coarser block.) Not inlined: the flux pass calls it
// from eight places per axis, and one shared copy keeps the pass's code in the instruction cache
// (inlined, instruction-fetch stalls led; the pass ran 4-7 % of the step slower).
template <int DIM, int R, bool ISEN>
__device__ __noinline__ void predict_texel(const KParams& P, const int* __restrict__ bt, const float4* __restrict__ w1,
                                              const float4* __restrict__ w2, int slot, const int* l0, float h, int axis,
                                              Pred& pr, float* su, float* sd, const int* __restrict__ bins = nullptr) {
  int l[3] = {l0[0], l0[1], l0[2]};
  float flip[3] = {1.f, 1.f, 1.f}, mask[3] = {1.f, 1.f, 1.f};
  int out = 0, oa = 0;
#pragma unroll
  for (int a = 0; a < DIM; a++)
    if (l[a] < 0 || l[a] >= BS) { out++; oa = a; }
  bool moved = false;
  if (out == 1) {
    const int upper = l[oa] >= BS ? 1 : 0;
    const int nb = bt_at(bt, slot, 6 + 2 * oa + upper);
    if (nb == -1 || (nb >= 0 && nb != slot && mid_block(bt, bins, nb))) {
#pragma unroll
      for (int a = 0; a < DIM; a++)
        if (a != oa) mask[a] = (l[a] == 0 || l[a] == BS - 1) ? 0.f : 1.f;
    } else if (nb <= -2) {
      if (-1 - nb == 2) {
        l[oa] = upper ? 2 * BS - 1 - l[oa] : -1 - l[oa];
        flip[oa] = -1.f;
      } else {
        l[oa] = upper ? BS - 1 : 0;
      }
      moved = true;
    }
  }
  float c[7], sua[DIM][6], sda[DIM][6];
  float conv = 0.f, jump = -INFINITY;
  load_w7<DIM>(w1, w2, slot, l, c);
#pragma unroll
  for (int a = 0; a < DIM; a++) {
    float m[7], p[7];
    int lm[3] = {l[0], l[1], l[2]}, lp[3] = {l[0], l[1], l[2]};
    lm[a] -= 1;
    lp[a] += 1;
    load_w6<DIM>(w1, w2, slot, lm, m);
    load_w6<DIM>(w1, w2, slot, lp, p);
    axis_edges<R, ISEN>(m, m, c, p, p, P.inv_gamma, sua[a], sda[a]);
    conv += p[1 + a] - m[1 + a];
    jump = fmaxf(jump, jump_excess(m[4], p[4], P.shock_thresh));
  }
  hancock_masked<DIM>(c, conv, jump, sua, sda, mask, h, P, pr);
  pr.q[1] *= flip[0];
  pr.q[2] *= flip[1];
  pr.q[3] *= flip[2];
  if (moved) {
    float g[7], m[7], p[7];
    int lm[3] = {l0[0], l0[1], l0[2]}, lp[3] = {l0[0], l0[1], l0[2]};
    lm[axis] -= 1;
    lp[axis] += 1;
    load_w7<DIM>(w1, w2, slot, l0, g);
    load_w6<DIM>(w1, w2, slot, lm, m);
    load_w6<DIM>(w1, w2, slot, lp, p);
    axis_edges<R, ISEN>(m, m, g, p, p, P.inv_gamma, su, sd);
  } else {
#pragma unroll
    for (int v = 0; v < 6; v++) {
      su[v] = sua[axis][v];
      sd[v] = sda[axis][v];
    }
  }
}

// The mean of the fine fluxes through the face of cell l on side `hi` of axis AXIS, whose
// same-level neighbour np is refined: computed from the fine leaf's own atlas as the fine leaf's
// sweep computes them.
struct Flux8 {
  float v[8];
};
// With per-block timesteps (bins) the fine leaf predicts with its own step (hf is the fine level's
// h for the clock's dt) and its fluxes count for their share of this block's step (kb, deposit:
// half for a faster child, none in a deposit for one in step; amr/update.wgsl:182-186).
template <int DIM, int R, bool ISEN, int AXIS>
__device__ __forceinline__ Flux8 fine_mean_flux(const KParams* __restrict__ Pp, const int* __restrict__ bt,
                                             const float4* __restrict__ w1, const float4* __restrict__ w2, int np, int l0,
                                             int l1, int l2, bool hi, float hf, const int* __restrict__ bins = nullptr,
                                             int kb = 0, bool deposit = false) {
  const KParams& P = *Pp;
  Flux8 out;
#pragma unroll
  for (int v = 0; v < 8; v++) out.v[v] = 0.f;
  const int l[3] = {l0, l1, l2};
  const bool upper = !hi;
  int hb[3] = {l[0] >= BS / 2, l[1] >= BS / 2, DIM == 3 ? (l[2] >= BS / 2) : 0};
  int bits[3] = {hb[0], hb[1], hb[2]};
  bits[AXIS] = upper ? 1 : 0;
  if (DIM == 2) bits[2] = 0;
  const int ch = bt_at(bt, np, 12 + (bits[0] | (bits[1] << 1) | (bits[2] << 2)));
  if (ch < 0) return out;
  float part = 1.f;
  if (bins) {
    const int kc = blk_bin(bins, ch);
    part = kc < kb ? 0.5f : (deposit ? 0.f : 1.f);
    if (part == 0.f) return out;
    hf *= (float)(1 << kc);
  }
  int a0[3] = {2 * (l[0] - (BS / 2) * hb[0]), 2 * (l[1] - (BS / 2) * hb[1]), DIM == 3 ? 2 * (l[2] - (BS / 2) * hb[2]) : 0};
  a0[AXIS] = upper ? BS - 1 : -1;
  constexpr int T1 = (AXIS + 1) % 3, T2 = (AXIS + 2) % 3;
  const int n1 = (DIM == 2 && T1 == 2) ? 1 : 2;
  const int n2 = (DIM == 2 && T2 == 2) ? 1 : 2;
  for (int j = 0; j < n2; j++)
    for (int i = 0; i < n1; i++) {
      int a[3] = {a0[0], a0[1], a0[2]};
      a[T1] += i;
      a[T2] += j;
      int b[3] = {a[0], a[1], a[2]};
      b[AXIS] += 1;
      Pred pa, pb;
      float sua[6], sda[6], sub[6], sdb[6];
      predict_texel<DIM, R, ISEN>(P, bt, w1, w2, ch, a, hf, AXIS, pa, sua, sda, bins);
      predict_texel<DIM, R, ISEN>(P, bt, w1, w2, ch, b, hf, AXIS, pb, sub, sdb, bins);
      float L[7], Rr[7], f[8];
      face_state(pa, sua, 1.f, L);
      face_state(pb, sdb, -1.f, Rr);
      riemann<AXIS>(L, Rr, P, f);
#pragma unroll
      for (int v = 0; v < 8; v++) out.v[v] += f[v];
    }
  float w = 1.f / (float)(n1 * n2);
  if (bins) w *= part;
#pragma unroll
  for (int v = 0; v < 8; v++) out.v[v] *= w;
  return out;
}

// Per-block timesteps: the flux through the face of cell (l0, l1, l2) on side `hi` of axis AXIS
// whose same-level neighbour np is a leaf in a faster bin, as np computes it with its own step
// (hn: np's h), for half of this block's step (amr/update.wgsl:253-256).
template <int DIM, int R, bool ISEN, int AXIS>
__device__ __forceinline__ Flux8 fast_face_flux(const KParams* __restrict__ Pp, const int* __restrict__ bt,
                                                const float4* __restrict__ w1, const float4* __restrict__ w2,
                                                const int* __restrict__ bins, int np, int l0, int l1, int l2, bool hi,
                                                float hn) {
  const KParams& P = *Pp;
  int a[3] = {l0, l1, l2};
  a[AXIS] = hi ? -1 : BS - 1;  // np lies above: its ghost below its first cell; below: its last cell
  int b[3] = {a[0], a[1], a[2]};
  b[AXIS] += 1;
  Pred pa, pb;
  float sua[6], sda[6], sub[6], sdb[6];
  predict_texel<DIM, R, ISEN>(P, bt, w1, w2, np, a, hn, AXIS, pa, sua, sda, bins);
  predict_texel<DIM, R, ISEN>(P, bt, w1, w2, np, b, hn, AXIS, pb, sub, sdb, bins);
  float L[7], Rr[7];
  Flux8 out;
  face_state(pa, sua, 1.f, L);
  face_state(pb, sdb, -1.f, Rr);
  riemann<AXIS>(L, Rr, P, out.v);
#pragma unroll
  for (int v = 0; v < 8; v++) out.v[v] *= 0.5f;
  return out;
}

// Fine-flux matching, ahead of the sweep (amr/update.wgsl:207-295): for every face of a leaf
// whose same-level neighbour is refined, the mean of the fine fluxes through each of its cells,
// into the buffer entry the host assigned (entries: leaf slot, face, index). One thread per face
// cell, so that the few blocks with such faces do not hold up a sweep's CTA.
// With per-block timesteps (bins) the list also holds, per substep, the faces of the leaves that
// update whose same-level neighbour is a leaf in a faster bin: that neighbour's own flux, half of
// it; and the refined neighbours' fluxes carry their children's shares.
template <int DIM, int R, bool ISEN>
__global__ void __launch_bounds__(NT) amr_fine_flux(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                    const int* __restrict__ flist, int nf, const float4* __restrict__ w1,
                                                    const float4* __restrict__ w2, const DevClock* __restrict__ clks,
                                                    float4* __restrict__ fbuf, const int* __restrict__ bins) {
  constexpr int FC = DIM == 3 ? BS * BS : BS;  // cells of a face
  const long long total = (long long)nf * FC;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(t / FC), c = (int)(t % FC);
    const int slot = __ldg(flist + 3 * e), f = __ldg(flist + 3 * e + 1), k = __ldg(flist + 3 * e + 2);
    const int g = bt_at(bt, slot, GRID_WORD);
    if (clks[g].held) continue;
    const KParams* Pp = gp + g;
    const double dt = clks[g].dt;
    const float hf = (float)((0.5 * dt) / (Pp->dx / ldexp(1.0, bt_at(bt, slot, 0) + 1)));  // h at the fine level
    const int axis = f >> 1;
    const bool hi = (f & 1) != 0;
    const int np = bt_at(bt, slot, 6 + f);
    const int t1 = c % BS, t2 = c / BS;
    const int edge = hi ? BS - 1 : 0;
    Flux8 F;
    if (bins && leaf_of(bt, np)) {
      const float hn = (float)((0.5 * (dt * ldexp(1.0, blk_bin(bins, np)))) / (Pp->dx / ldexp(1.0, bt_at(bt, slot, 0))));
      if (axis == 0) F = fast_face_flux<DIM, R, ISEN, 0>(Pp, bt, w1, w2, bins, np, edge, t1, t2, hi, hn);
      else if (axis == 1) F = fast_face_flux<DIM, R, ISEN, 1>(Pp, bt, w1, w2, bins, np, t1, edge, t2, hi, hn);
      else F = fast_face_flux<DIM, R, ISEN, 2>(Pp, bt, w1, w2, bins, np, t1, t2, edge, hi, hn);
    } else {
      const int kb = blk_bin(bins, slot);
      const bool dep = !blk_active(bins, slot);
      if (axis == 0) F = fine_mean_flux<DIM, R, ISEN, 0>(Pp, bt, w1, w2, np, edge, t1, t2, hi, hf, bins, kb, dep);
      else if (axis == 1) F = fine_mean_flux<DIM, R, ISEN, 1>(Pp, bt, w1, w2, np, t1, edge, t2, hi, hf, bins, kb, dep);
      else F = fine_mean_flux<DIM, R, ISEN, 2>(Pp, bt, w1, w2, np, t1, t2, edge, hi, hf, bins, kb, dep);
    }
    float4* o = fbuf + ((size_t)k * FC + c) * 2;
    o[0] = make_float4(F.v[0], F.v[1], F.v[2], F.v[3]);
    o[1] = make_float4(F.v[4], F.v[5], F.v[6], F.v[7]);
  }
}

// Shared memory of the block sweep, in floats. The primitive planes are a ring of three, each the
// plane's w1 texels then its w2 texels (float4, as in the atlas), filled by bulk copies (TMA): the
// predictor at plane j reads planes j - 1, j, j + 1; once every thread is past it, plane j - 1's
// slot takes plane j + 2, in flight during the fluxes and updates of plane j. (A fourth slot, for
// a copy issued a plane earlier, would leave no room for the flux sums held here instead of in
// registers at two CTAs per SM.)
constexpr int RING = 3;
constexpr int SW_PLANE = 2 * 4 * SWN;    // floats of one staged plane (w1 and w2)
constexpr int SW_RING = RING * SW_PLANE;
constexpr int SW_FACE = 2 * 7 * SPN;  // x and y upper face states of a plane
constexpr int SW_FLUX = 2 * 8 * SPN;  // x and y lower-face fluxes of a plane (also the half-step exchange)
constexpr int SW_KEEP = 8 * SPN;      // z boundary ghosts: a plane's half steps or the ghost's increments
constexpr int SW_ZUP = 7 * SPN;       // each thread's upper z face state, for the next plane's z face
constexpr int SW_ACC = 8 * SPN;       // each thread's flux sums of the plane below, until its upper z face
constexpr size_t SWEEP_SMEM = (size_t)(SW_RING + SW_FACE + SW_FLUX + SW_KEEP + SW_ZUP + SW_ACC) * sizeof(float);
constexpr uint32_t PLANE_BYTES = SWN * sizeof(float4);  // one of w1 / w2 of a plane: 6400 B

// Texel (x, y) of a staged plane: its seven primitives (the sound speed as the atlas holds it).
__device__ __forceinline__ void read_w7(const float4* __restrict__ plane, int x, int y, float* w) {
  const int t = (y + NG) * PAD + (x + NG);
  const float4 a = plane[t], b = plane[SWN + t];
  w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
  w[4] = b.x; w[5] = b.y; w[6] = b.z;
}

// Per-block timesteps (bins, the bin table; null: one timestep): each block steps with its own
// 2^k dt; a ghost beside a neighbour part way through its step (whose ghosts the assemble filled
// from its half step) is predicted in place, as beside a coarser block; faces whose same-level
// neighbour is a faster leaf also take their flux from the buffer (entries from fbase[slot], per
// substep); a block in a bin above 0 keeps its half steps (block and first ghost layer) in p1, p2
// for its neighbours' ghosts and its own deposits while it is part way through its step. The
// state is then updated in place (o1, o2 the arrays u1, u2): each cell is read once, by the
// thread that writes it, and no other pass of the launch reads the state.
template <int DIM, int R, bool ISEN, bool BINS>
__global__ void __maxnreg__(80)
    amr_sweep(const KParams* __restrict__ gp, const int* __restrict__ bt, const int* __restrict__ list, int n,
              const float4* __restrict__ u1, const float4* __restrict__ u2, const float4* __restrict__ w1,
              const float4* __restrict__ w2, float4* __restrict__ o1, float4* __restrict__ o2,
              const DevClock* __restrict__ clks, const float4* __restrict__ fbuf, int* __restrict__ err,
              const int* __restrict__ bins, const int* __restrict__ fbase, float4* __restrict__ p1,
              float4* __restrict__ p2) {
  constexpr int FC = DIM == 3 ? BS * BS : BS;  // cells of a face
  extern __shared__ __align__(128) float smem[];
  float* sW = smem;
  float* sFace = sW + SW_RING;
  float* sFlux = sFace + SW_FACE;
  float* sKeep = sFlux + SW_FLUX;
  float* sZup = sKeep + SW_KEEP;
  float* sAcc = sZup + SW_ZUP;
  // the block's grid parameters, copied once per block: the march reads them at every face
  __shared__ __align__(16) KParams sP;
  const int tid = threadIdx.x;
  const int tx = tid % SX, ty = tid / SX;
  const int lx = tx - 1, ly = DIM >= 2 ? ty - 1 : 0;
  const bool row_t = ty >= 1 && ty <= BS;
  const bool col_t = tx >= 1 && tx <= BS;
  const bool tile_t = row_t && col_t;
  auto ring = [&](int plane) -> const float4* {
    return reinterpret_cast<const float4*>(sW + (size_t)((plane + 3 * RING) % RING) * SW_PLANE);
  };
  // One mbarrier per ring slot; the phase each thread expects next, per slot (uniform across the
  // CTA: every thread waits for every plane once); slots with a copy in flight.
  __shared__ __align__(8) uint64_t sBar[RING];
  uint32_t phase = 0, pending = 0;
  if (tid == 0) {
    for (int s = 0; s < RING; s++) tma::mbar_init(&sBar[s], 1);
    tma::fence_mbar_init();
  }
  __syncthreads();

  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int slot = __ldg(list + i);
    const int g = bt_at(bt, slot, GRID_WORD);
    const int kb = BINS ? blk_bin(bins, slot) : 0;
    const double dt = BINS ? clks[g].dt * ldexp(1.0, kb) : clks[g].dt;
    const double dxl = gp[g].dx / ldexp(1.0, bt_at(bt, slot, 0));
    const float dtdx = (float)(dt / dxl);
    const float h = (float)((0.5 * dt) / dxl);
    const size_t base = (size_t)slot * BG<DIM>::CB;
    if (clks[g].held) {
      for (int t = tid; t < BG<DIM>::CB; t += SNT) {
        o1[base + t] = __ldg(u1 + base + t);
        o2[base + t] = __ldg(u2 + base + t);
      }
      continue;
    }
    __syncthreads();  // the previous block's last reads of shared memory
    static_assert(sizeof(KParams) % 4 == 0, "KParams is copied as words");
    if (tid < (int)(sizeof(KParams) / 4))
      reinterpret_cast<int*>(&sP)[tid] = __ldg(reinterpret_cast<const int*>(gp + g) + tid);
    const KParams& P = sP;
    // This thread's ghost role across x or y: the face and, for a domain boundary, the thread
    // holding the inner cell that the ghost maps to (mirror or edge cell: both the adjacent one).
    int gface = -1;
    if (tx == 0 && row_t) gface = 0;
    if (tx == SX - 1 && row_t) gface = 1;
    if (DIM >= 2 && ty == 0 && col_t) gface = 2;
    if (DIM >= 2 && ty == SX - 1 && col_t) gface = 3;
    const int gnb = gface >= 0 ? bt_at(bt, slot, 6 + gface) : 0;
    const bool g_coarse = gface >= 0 && (gnb == -1 || (BINS && gnb >= 0 && gnb != slot && mid_block(bt, bins, gnb)));
    const bool g_bc = gface >= 0 && gnb <= -2;
    const int g_src = !g_bc ? -1 : (gface == 0 ? tid + 1 : gface == 1 ? tid - 1 : gface == 2 ? tid + SX : tid - SX);
    const bool g_flip = g_bc && (-1 - gnb) == 2;
    const int g_axis = gface >> 1;
    bool xyg = false;
#pragma unroll
    for (int f = 0; f < 4; f++) xyg = xyg || bt_at(bt, slot, 6 + f) <= -2;
    // the faces' fine-flux matching (a same-level neighbour that is refined): their fluxes are
    // in the buffer, from amr_fine_flux, at entries fine0 on in face order
    unsigned fine = 0;
#pragma unroll
    for (int f = 0; f < 2 * DIM; f++) {
      const int nb = bt_at(bt, slot, 6 + f);
      if (nb >= 0 && !leaf_of(bt, nb)) fine |= 1u << f;
      else if (BINS && nb >= 0 && nb != slot && blk_bin(bins, nb) < kb) fine |= 1u << f;
    }
    const int fine0 = BINS ? __ldg(fbase + slot) : bt_at(bt, slot, FINE_WORD);
    if (fine0 < 0 || fbuf == nullptr) fine = 0;
    auto matched = [&](int f, int cidx, float* F) {
      const float4* q = fbuf + ((size_t)(fine0 + __popc(fine & ((1u << f) - 1u))) * FC + cidx) * 2;
      const float4 a = __ldg(q), b = __ldg(q + 1);
      F[0] = a.x; F[1] = a.y; F[2] = a.z; F[3] = a.w;
      F[4] = b.x; F[5] = b.y; F[6] = b.z; F[7] = b.w;
    };
    const int zlo_nb = DIM == 3 ? bt_at(bt, slot, 10) : 0, zhi_nb = DIM == 3 ? bt_at(bt, slot, 11) : 0;
    // z ghosts predicted in place: beside a coarser block or one part way through its step
    const bool zlo_in = DIM == 3 && (zlo_nb == -1 || (BINS && zlo_nb >= 0 && zlo_nb != slot && mid_block(bt, bins, zlo_nb)));
    const bool zhi_in = DIM == 3 && (zhi_nb == -1 || (BINS && zhi_nb >= 0 && zhi_nb != slot && mid_block(bt, bins, zhi_nb)));
    const bool keep = BINS && kb > 0;  // this block's half steps are kept
    auto keep_pred = [&](int lz, const Pred& q) {
      const int l[3] = {lx, ly, lz};
      const size_t o = (size_t)slot * BG<DIM>::PN + ptex<DIM>(l);
      p1[o] = make_float4(q.q[0], q.q[1], q.q[2], q.q[3]);
      p2[o] = make_float4(q.q[4], q.q[5], q.flag, q.fo ? 1.f : 0.f);
    };

    float ph_prev = 0.f;
    // CTA-uniform: a predicted cell of plane j - 1 (block and ghost ring) is shock-flagged. The
    // faces of plane j see the flags of planes j - 1 and j only; without any, the solver skips the
    // HLL flux.
    bool flagged_prev = true;

    // Plane pl (-2 .. 17) of this block's atlas into its ring slot: issued by one thread, after a
    // barrier that follows every thread's last read of the slot (the plane three before).
    auto issue = [&](int pl) {
      const int s = (pl + 3 * RING) % RING;
      if (tid == 0) {
        const size_t zb = (size_t)slot * BG<DIM>::WN + (DIM == 3 ? (size_t)(pl + NG) * SWN : 0);
        float4* dst = reinterpret_cast<float4*>(sW + (size_t)s * SW_PLANE);
        tma::fence_proxy_async();
        tma::mbar_expect_tx(&sBar[s], 2 * PLANE_BYTES);
        tma::bulk_g2s(dst, w1 + zb, PLANE_BYTES, &sBar[s]);
        tma::bulk_g2s(dst + SWN, w2 + zb, PLANE_BYTES, &sBar[s]);
      }
      pending |= 1u << s;
    };
    // Wait for plane pl; CTA-uniformly false if the copy did not complete in time.
    auto arrived = [&](int pl) -> bool {
      const int s = (pl + 3 * RING) % RING;
      const bool ok = tma::mbar_wait(&sBar[s], (phase >> s) & 1u, tma::WAIT_LIMIT);
      phase ^= 1u << s;
      pending &= ~(1u << s);
      return !__syncthreads_or(!ok);
    };
    // A copy that never completed: record it, let the others land (bounded), leave.
    auto give_up = [&]() {
      if (tid == 0 && err) atomicExch(err, tma::ERR_TMA_TIMEOUT);
      for (int s = 0; s < RING; s++)
        if (pending & (1u << s)) tma::mbar_wait(&sBar[s], (phase >> s) & 1u, tma::WAIT_LIMIT);
    };
    if constexpr (DIM == 3) {
      issue(-2);
      issue(-1);
      issue(0);
      if (!arrived(-2) || !arrived(-1)) {
        give_up();
        return;
      }
    } else {
      issue(0);
    }
    // 3D: planes -1 .. 16, the first and last the z ghosts; 2D: the one plane.
    const int jb = DIM == 3 ? -1 : 0, je = DIM == 3 ? BS : 0;
    for (int j = jb; j <= je; j++) {
      if (!arrived(DIM == 3 ? j + 1 : 0)) {
        give_up();
        return;
      }
      const float4* pj = ring(DIM == 3 ? j : 0);
      const bool zghost = DIM == 3 && (j == -1 || j == BS);

      // the predictor at plane j
      float c[7];
      read_w7(pj, lx, ly, c);
      float su[DIM][6], sd[DIM][6];
      float conv = 0.f, jump = -INFINITY;
      {
        float m[7], p[7];
        read_w7(pj, lx - 1, ly, m);
        read_w7(pj, lx + 1, ly, p);
        axis_edges<R, ISEN>(m, m, c, p, p, P.inv_gamma, su[0], sd[0]);
        conv += p[1] - m[1];
        jump = fmaxf(jump, jump_excess(m[4], p[4], P.shock_thresh));
        if constexpr (DIM >= 2) {
          read_w7(pj, lx, ly - 1, m);
          read_w7(pj, lx, ly + 1, p);
          axis_edges<R, ISEN>(m, m, c, p, p, P.inv_gamma, su[1], sd[1]);
          conv += p[2] - m[2];
          jump = fmaxf(jump, jump_excess(m[4], p[4], P.shock_thresh));
        }
        if constexpr (DIM == 3) {
          read_w7(ring(j - 1), lx, ly, m);
          read_w7(ring(j + 1), lx, ly, p);
          axis_edges<R, ISEN>(m, m, c, p, p, P.inv_gamma, su[2], sd[2]);
          conv += p[3] - m[3];
          jump = fmaxf(jump, jump_excess(m[4], p[4], P.shock_thresh));
        }
      }
      // a ghost beside a coarser block: the slopes along the face's transverse axes dropped at
      // the rim of the face
      float mask[3] = {1.f, 1.f, 1.f};
      {
        const int lz = DIM == 3 ? j : 0;
        const float rx = (lx == 0 || lx == BS - 1) ? 0.f : 1.f;
        const float ry = (ly == 0 || ly == BS - 1) ? 0.f : 1.f;
        const float rz = (lz == 0 || lz == BS - 1) ? 0.f : 1.f;
        if (zghost && (j == -1 ? zlo_in : zhi_in)) {
          mask[0] = rx;
          mask[1] = ry;
        } else if (g_coarse) {
          if (g_axis == 0) mask[1] = ry;
          else mask[0] = rx;
          if (DIM == 3) mask[2] = rz;
        }
      }
      Pred pr;
      hancock_masked<DIM>(c, conv, jump, su, sd, mask, h, P, pr);

      const bool tile_plane = j >= 0 && j < (DIM == 3 ? BS : 1);
      if (xyg && tile_plane) {
        // x and y boundary ghosts take the half step of the inner cell they map to
#pragma unroll
        for (int v = 0; v < 6; v++) sFlux[v * SPN + tid] = pr.q[v];
        sFlux[6 * SPN + tid] = pr.flag;
        sFlux[7 * SPN + tid] = pr.fo ? 1.f : 0.f;
        __syncthreads();
        if (g_src >= 0) {
#pragma unroll
          for (int v = 0; v < 6; v++) pr.q[v] = sFlux[v * SPN + g_src];
          if (g_flip) pr.q[1 + g_axis] = -pr.q[1 + g_axis];
          pr.flag = sFlux[6 * SPN + g_src];
          pr.fo = sFlux[7 * SPN + g_src] != 0.f;
        }
      }
      if constexpr (DIM == 3) {
        // z boundary ghosts: the lower one takes plane 0's half step with its own increments
        // (kept from plane -1); the upper one plane 15's (kept from plane 15). Each thread keeps
        // and reads back its own column: no barrier needed.
        if (j == -1 && zlo_nb <= -2) {
#pragma unroll
          for (int v = 0; v < 6; v++) sKeep[v * SPN + tid] = su[2][v];
        }
        if (j == 0 && zlo_nb <= -2) {
          Pred gq = pr;
          if (-1 - zlo_nb == 2) gq.q[3] = -gq.q[3];
          float inc[6];
#pragma unroll
          for (int v = 0; v < 6; v++) inc[v] = sKeep[v * SPN + tid];
          float zf[7];
          face_state(gq, inc, 1.f, zf);
#pragma unroll
          for (int q = 0; q < 7; q++) sZup[q * SPN + tid] = zf[q];
          if (keep) keep_pred(-1, gq);  // the lower boundary ghost: plane 0's half step, mirrored
        }
        if (j == BS - 1 && zhi_nb <= -2) {
#pragma unroll
          for (int v = 0; v < 6; v++) sKeep[v * SPN + tid] = pr.q[v];
          sKeep[6 * SPN + tid] = pr.flag;
          sKeep[7 * SPN + tid] = pr.fo ? 1.f : 0.f;
        }
        if (j == BS && zhi_nb <= -2) {
#pragma unroll
          for (int v = 0; v < 6; v++) pr.q[v] = sKeep[v * SPN + tid];
          if (-1 - zhi_nb == 2) pr.q[3] = -pr.q[3];
          pr.flag = sKeep[6 * SPN + tid];
          pr.fo = sKeep[7 * SPN + tid] != 0.f;
        }
      }
      if (keep && !(DIM == 3 && j == -1 && zlo_nb <= -2)) keep_pred(DIM == 3 ? j : 0, pr);
      if (tile_plane) {
        float f[7];
        face_state(pr, su[0], 1.f, f);
#pragma unroll
        for (int v = 0; v < 7; v++) sFace[v * SPN + tid] = f[v];
        if constexpr (DIM >= 2) {
          face_state(pr, su[1], 1.f, f);
#pragma unroll
          for (int v = 0; v < 7; v++) sFace[(7 + v) * SPN + tid] = f[v];
        }
      }
      const bool flagged = __syncthreads_or(pr.flag != 0.f);
      const bool hll_any = flagged || (DIM == 3 && flagged_prev);
      flagged_prev = flagged;
      // every thread is done with plane j - 1: its ring slot takes plane j + 2
      if (DIM == 3 && j + 2 <= BS + 1) issue(j + 2);

      const int lz = DIM == 3 ? j : 0;
      if (tile_plane) {
        if (row_t && tx >= 1) {
          // the x face below cell lx (lx = 0 .. 16)
          float L[7], Rr[7], F[8];
#pragma unroll
          for (int v = 0; v < 7; v++) L[v] = sFace[v * SPN + tid - 1];
          face_state(pr, sd[0], -1.f, Rr);
          riemann<0>(L, Rr, P, F, hll_any);
          if ((lx == 0 && (fine & 1u)) || (lx == BS && (fine & 2u))) matched(lx == 0 ? 0 : 1, ly + BS * lz, F);
#pragma unroll
          for (int v = 0; v < 8; v++) sFlux[v * SPN + tid] = F[v];
        }
        if constexpr (DIM >= 2) {
          if (col_t && ty >= 1) {
            float L[7], Rr[7], F[8];
#pragma unroll
            for (int v = 0; v < 7; v++) L[v] = sFace[(7 + v) * SPN + tid - SX];
            face_state(pr, sd[1], -1.f, Rr);
            riemann<1>(L, Rr, P, F, hll_any);
            if ((ly == 0 && (fine & 4u)) || (ly == BS && (fine & 8u))) matched(ly == 0 ? 2 : 3, lx + BS * lz, F);
#pragma unroll
            for (int v = 0; v < 8; v++) sFlux[(8 + v) * SPN + tid] = F[v];
          }
        }
      }
      float Fz[8];
      if constexpr (DIM == 3) {
        if (tile_t && j >= 0) {
          // the z face below plane j
          float Rr[7];
          face_state(pr, sd[2], -1.f, Rr);
          float zf[7];
#pragma unroll
          for (int q = 0; q < 7; q++) zf[q] = sZup[q * SPN + tid];
          riemann<2>(zf, Rr, P, Fz, hll_any);
          if ((j == 0 && (fine & 16u)) || (j == BS && (fine & 32u))) matched(j == 0 ? 4 : 5, lx + BS * ly, Fz);
        }
      }
      __syncthreads();

      if (tile_t) {
        float acc[8];
        if constexpr (DIM == 3) {
          if (j >= 1) {
            // plane j - 1 is complete: its upper z face is Fz
#pragma unroll
            for (int v = 0; v < 8; v++) acc[v] = sAcc[v * SPN + tid] - Fz[v];
            const size_t o = base + ((size_t)(j - 1) * BS + ly) * BS + lx;
            float4 na, nb4;
            update_cell(__ldg(u1 + o), __ldg(u2 + o), acc, ph_prev, dtdx, P, na, nb4);
            o1[o] = na;
            o2[o] = nb4;
          }
        }
        if (tile_plane) {
#pragma unroll
          for (int v = 0; v < 8; v++) {
            float a = sFlux[v * SPN + tid];
            a -= sFlux[v * SPN + tid + 1];
            if constexpr (DIM >= 2) {
              a += sFlux[(8 + v) * SPN + tid];
              a -= sFlux[(8 + v) * SPN + tid + SX];
            }
            if constexpr (DIM == 3) {
              a += Fz[v];
              sAcc[v * SPN + tid] = a;
            } else {
              acc[v] = a;
            }
          }
          ph_prev = pr.q[4];
          if constexpr (DIM < 3) {
            const size_t o = base + (size_t)ly * BS + lx;
            float4 na, nb4;
            update_cell(__ldg(u1 + o), __ldg(u2 + o), acc, ph_prev, dtdx, P, na, nb4);
            o1[o] = na;
            o2[o] = nb4;
          }
        }
      }
      if constexpr (DIM == 3) {
        // the upper z face state of plane j (a lower boundary ghost's is set at plane 0)
        if (!(j == -1 && zlo_nb <= -2)) {
          float zf[7];
          face_state(pr, su[2], 1.f, zf);
#pragma unroll
          for (int q = 0; q < 7; q++) sZup[q * SPN + tid] = zf[q];
        }
      }
    }
  }
}

// Per-block timesteps, the deposit (amr/update.wgsl:339-445 with g_deposit): a leaf half way
// through its step beside a faster neighbour takes, on the cells of the shared faces, that
// neighbour's fluxes of its second step for half of this block's step (from the buffer the
// neighbour-flux pass filled), with the half-step pressure its own prediction kept from the start
// of its step; no fluxes of its own. Cells on no such face keep their state. In place.
template <int DIM>
__global__ void __launch_bounds__(NT) amr_deposit(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                  const int* __restrict__ list, int n, float4* __restrict__ u1,
                                                  float4* __restrict__ u2, const float4* __restrict__ p2,
                                                  const DevClock* __restrict__ clks, const int* __restrict__ bins,
                                                  const int* __restrict__ fbase, const float4* __restrict__ fbuf) {
  constexpr int FC = DIM == 3 ? BS * BS : BS;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int slot = __ldg(list + i);
    const int g = bt_at(bt, slot, GRID_WORD);
    if (clks[g].held) continue;
    const KParams& P = gp[g];
    const int kb = blk_bin(bins, slot);
    const double dt = clks[g].dt * ldexp(1.0, kb);
    const float dtdx = (float)(dt / (P.dx / ldexp(1.0, bt_at(bt, slot, 0))));
    unsigned fine = 0;
    for (int f = 0; f < 2 * DIM; f++) {
      const int nb = bt_at(bt, slot, 6 + f);
      if (nb >= 0 && !leaf_of(bt, nb)) fine |= 1u << f;
      else if (nb >= 0 && nb != slot && blk_bin(bins, nb) < kb) fine |= 1u << f;
    }
    const int fine0 = __ldg(fbase + slot);
    if (!fine || fine0 < 0) continue;
    for (int t = threadIdx.x; t < BG<DIM>::CB; t += NT) {
      const int l[3] = {t % BS, (t / BS) % BS, DIM == 3 ? t / (BS * BS) : 0};
      float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      bool touched = false;
      for (int f = 0; f < 2 * DIM; f++) {
        if (!(fine & (1u << f))) continue;
        const int axis = f >> 1;
        const bool hi = (f & 1) != 0;
        if (l[axis] != (hi ? BS - 1 : 0)) continue;
        const int nb = bt_at(bt, slot, 6 + f);
        if (!leaf_of(bt, nb)) {
          // the refined neighbour's child on this cell's face: only a faster one gives a deposit
          int bits[3] = {l[0] >= BS / 2, l[1] >= BS / 2, DIM == 3 ? (l[2] >= BS / 2) : 0};
          bits[axis] = hi ? 0 : 1;
          const int ch = bt_at(bt, nb, 12 + (bits[0] | (bits[1] << 1) | (bits[2] << 2)));
          if (ch < 0 || blk_bin(bins, ch) >= kb) continue;
        }
        touched = true;
        const int cidx = axis == 0 ? l[1] + BS * l[2] : axis == 1 ? l[0] + BS * l[2] : l[0] + BS * l[1];
        const float4* q = fbuf + ((size_t)(fine0 + __popc(fine & ((1u << f) - 1u))) * FC + cidx) * 2;
        const float4 a = __ldg(q), b = __ldg(q + 1);
        const float F[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int v = 0; v < 8; v++) acc[v] = hi ? acc[v] - F[v] : acc[v] + F[v];
      }
      if (!touched) continue;
      const size_t o = (size_t)slot * BG<DIM>::CB + t;
      const float ph = __ldg(p2 + (size_t)slot * BG<DIM>::PN + ptex<DIM>(l)).x;
      float4 na, nb4;
      update_cell(u1[o], u2[o], acc, ph, dtdx, P, na, nb4);
      u1[o] = na;
      u2[o] = nb4;
    }
  }
}

}  // namespace amrk

// Host launchers.

namespace {
template <int DIM, int R, bool ISEN, bool BINS>
cudaError_t sweep_one(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, float4* o1,
                      float4* o2, const DevClock* clks, cudaStream_t s, int per_sm) {
  auto k = amrk::amr_sweep<DIM, R, ISEN, BINS>;
  // (set once per instantiation; an attribute call is not a stream operation, so a first call
  // inside a stream capture is fine)
  static const cudaError_t attr = [&] {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)amrk::SWEEP_SMEM);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    return e;
  }();
  if (attr != cudaSuccess) return attr;
  k<<<grid_for(n, per_sm), amrk::SNT, amrk::SWEEP_SMEM, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, o1, o2, clks, L.fbuf,
                                                             L.err, L.bins, L.fbase, L.p1, L.p2);
  return cudaGetLastError();
}
}  // namespace

cudaError_t amr_launch_fine_flux(const AmrLaunch& L, const int* flist, int nf, const DevClock* clks, cudaStream_t s,
                                 const tune::Choice* c) {
  if (nf <= 0) return cudaSuccess;
  const long long cells = (long long)nf * (L.ndim == 3 ? 256 : 16);
  const int per_sm = c && c->per_sm > 0 ? c->per_sm : 8;
  const int g = (int)std::min<long long>((cells + amrk::NT - 1) / amrk::NT, 148LL * per_sm);
  if (L.ndim == 3) {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_fine_flux<3, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, flist, nf, L.w1, L.w2, clks, L.fbuf, L.bins))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_fine_flux<3, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, flist, nf, L.w1, L.w2, clks, L.fbuf, L.bins))) }
  } else {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_fine_flux<2, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, flist, nf, L.w1, L.w2, clks, L.fbuf, L.bins))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_fine_flux<2, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, flist, nf, L.w1, L.w2, clks, L.fbuf, L.bins))) }
  }
  return cudaGetLastError();
}

cudaError_t amr_launch_deposit(const AmrLaunch& L, const int* list, int n, float4* u1, float4* u2, const DevClock* clks,
                               cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int g = grid_for(n, 4);
  if (L.ndim == 3) amrk::amr_deposit<3><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.p2, clks, L.bins, L.fbase, L.fbuf);
  else amrk::amr_deposit<2><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.p2, clks, L.bins, L.fbase, L.fbuf);
  return cudaGetLastError();
}

cudaError_t amr_launch_sweep(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, float4* o1,
                             float4* o2, const DevClock* clks, cudaStream_t s, const tune::Choice* c) {
  if (n <= 0) return cudaSuccess;
  const int per_sm = c && c->per_sm > 0 ? c->per_sm : 2;
  // (per-block timesteps in their own instantiation: the plain sweep's registers stay its own)
  if (L.bins) {
    if (L.ndim == 3) {
      if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, return (sweep_one<3, R, true, true>(L, list, n, u1, u2, o1, o2, clks, s, per_sm))) }
      else { SHZ_RECON_SWITCH(L.recon, false, return (sweep_one<3, R, false, true>(L, list, n, u1, u2, o1, o2, clks, s, per_sm))) }
    } else {
      if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, return (sweep_one<2, R, true, true>(L, list, n, u1, u2, o1, o2, clks, s, per_sm))) }
      else { SHZ_RECON_SWITCH(L.recon, false, return (sweep_one<2, R, false, true>(L, list, n, u1, u2, o1, o2, clks, s, per_sm))) }
    }
    return cudaSuccess;
  }
  if (L.ndim == 3) {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, return (sweep_one<3, R, true, false>(L, list, n, u1, u2, o1, o2, clks, s, per_sm))) }
    else { SHZ_RECON_SWITCH(L.recon, false, return (sweep_one<3, R, false, false>(L, list, n, u1, u2, o1, o2, clks, s, per_sm))) }
  } else {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, return (sweep_one<2, R, true, false>(L, list, n, u1, u2, o1, o2, clks, s, per_sm))) }
    else { SHZ_RECON_SWITCH(L.recon, false, return (sweep_one<2, R, false, false>(L, list, n, u1, u2, o1, o2, clks, s, per_sm))) }
  }
  return cudaSuccess;
}

}  // namespace shz

// ---------------------------------------------------------------------------------------------
// Tuned launches of the block kernels.

namespace shz {

tune::Key amr_tune_key(int kernel, const AmrLaunch& L, long long units) {
  const int isen = (kernel == tune::K_AMR_ASSEMBLE || kernel == tune::K_AMR_ASSEMBLE_BINS) ? 0 : (L.isen ? 1 : 0);
  return tune::Key{kernel, L.ndim, L.recon, isen, tune::size_class(units)};
}

namespace {
cudaError_t run_tuned(const tune::Key& k, const std::vector<tune::Choice>& cands, bool tune_now, cudaStream_t s,
                      const std::function<cudaError_t(const tune::Choice*)>& launch, long long* launches) {
  tune::Choice c;
  if (tune::pinned(k.kernel, &c) || tune::lookup(k, &c)) {
    *launches += 1;
    return launch(&c);
  }
  if (!tune_now || !tune::enabled()) {
    *launches += 1;
    return launch(nullptr);
  }
  const int reps = 2;
  *launches += (long long)cands.size() * (1 + reps);
  return tune::choose(k, cands, [&](const tune::Choice& x) { return launch(&x); }, s, reps, &c);
}
tune::Choice mk(int variant, int per_sm) {
  tune::Choice c;
  c.variant = variant;
  c.per_sm = per_sm;
  return c;
}
}  // namespace

cudaError_t amr_assemble_tuned(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                               unsigned* rates, int rslot, cudaStream_t s, bool tune_now, long long* launches) {
  if (n <= 0) return cudaSuccess;
  std::vector<tune::Choice> cands;
  for (int v : {0, 1, 2})
    for (int p : {4, 2, 8}) cands.push_back(mk(v, p));
  // the split form (variants 3, 4): the plain pass, then the rest at 2 or 3 CTAs' register budget;
  // (5, 6) the same two passes side by side, the second at 1 CTA an SM beside the first's 2
  for (int v : {3, 4})
    for (int p : {2, 4}) cands.push_back(mk(v, p));
  if (L.side) {
    cands.push_back(mk(5, 1));
    cands.push_back(mk(6, 1));
  }
  long long second = 0;  // the split form's second kernels (when the host listed blocks for them)
  const cudaError_t e = run_tuned(amr_tune_key(tune::K_AMR_ASSEMBLE, L, n), cands, tune_now, s,
                                  [&](const tune::Choice* c) {
                                    if (c && c->variant >= 3 && L.nrest != 0) second++;
                                    return amr_launch_assemble(L, list, n, u1, u2, rates, rslot, s, c);
                                  },
                                  launches);
  *launches += second;
  return e;
}

cudaError_t amr_assemble_bins_tuned(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                                    const int* bins, unsigned* rates, int rslot, float* brate, cudaStream_t s,
                                    long long* extra) {
  if (n <= 0) return cudaSuccess;
  const std::vector<tune::Choice> cands = {mk(1, 4), mk(3, 4), mk(3, 2)};
  long long launched = 0, second = 0;
  const cudaError_t e = run_tuned(amr_tune_key(tune::K_AMR_ASSEMBLE_BINS, L, n), cands, true, s,
                                  [&](const tune::Choice* c) {
                                    if (c && c->variant == 3) second++;
                                    return amr_launch_assemble_bins(L, list, n, u1, u2, bins, rates, rslot, brate, s, c);
                                  },
                                  &launched);
  *extra += launched - 1 + second;
  return e;
}

cudaError_t amr_fine_flux_tuned(const AmrLaunch& L, const int* flist, int nf, const DevClock* clks, cudaStream_t s,
                                bool tune_now, long long* launches) {
  if (nf <= 0) return cudaSuccess;
  const std::vector<tune::Choice> cands = {mk(0, 8), mk(0, 4), mk(0, 16)};
  return run_tuned(amr_tune_key(tune::K_AMR_FINE_FLUX, L, nf), cands, tune_now, s,
                   [&](const tune::Choice* c) { return amr_launch_fine_flux(L, flist, nf, clks, s, c); }, launches);
}

cudaError_t amr_sweep_tuned(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, float4* o1,
                            float4* o2, const DevClock* clks, cudaStream_t s, bool tune_now, long long* launches) {
  if (n <= 0) return cudaSuccess;
  const std::vector<tune::Choice> cands = {mk(0, 2), mk(0, 1), mk(0, 3), mk(0, 4)};
  return run_tuned(amr_tune_key(tune::K_AMR_SWEEP, L, n), cands, tune_now, s,
                   [&](const tune::Choice* c) { return amr_launch_sweep(L, list, n, u1, u2, o1, o2, clks, s, c); },
                   launches);
}

bool amr_step_wants_tuning(const AmrLaunch& L, int n_assembled, int n_leaves, int nf) {
  if (!tune::enabled()) return false;
  return (n_assembled > 0 && tune::needs(amr_tune_key(tune::K_AMR_ASSEMBLE, L, n_assembled))) ||
         (n_leaves > 0 && tune::needs(amr_tune_key(tune::K_AMR_SWEEP, L, n_leaves))) ||
         (nf > 0 && tune::needs(amr_tune_key(tune::K_AMR_FINE_FLUX, L, nf)));
}

}  // namespace shz
