// Device helpers shared by the adaptive-grid passes (amr_kernels.cu, amr_sweep.cu,
// amr_twopass.cu): block addressing, the ghost-source rule, restriction and prolongation, block
// maxima; and the host-side launch helpers.
//
// A block holds 16^ndim cells. Atlases live in HBM, slot-major, with x fastest:
//   - the conserved state: two parities of 16^ndim cells x (u1, u2) float4;
//   - the primitives with two ghost layers: 20^ndim cells x (w1 = rho, v; w2 = p, s, cs, 0);
//   - with two_pass only, the half-step states over the block and one ghost layer: 18^ndim cells
//     x (p1 = rho, v; p2 = p, s, shock flag, first-order flag).
// They follow the reference's rules for the ghost fill (amr/grid.wgsl:186-222 ghost_src;
// amr/cons.wgsl:19-125 restriction and prolongation; amr/assemble.wgsl:47-75 from_coarse).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "amr_kernels.h"
#include "hydro_cell.cuh"
#include "hydro_math.cuh"

namespace shz {
namespace amrk {


constexpr int BS = 16, NG = 2, PAD = BS + 2 * NG, PP = BS + 2, BTS = 32, RGS = 12;
// Word of a block-table row that holds the block's grid: an index into the per-grid parameters
// and clocks (a batch advances blocks of many independent grids in one pass).
constexpr int GRID_WORD = 26;
// Word of a leaf's row that holds the index of its first matched face in the fine-flux buffer
// (faces whose same-level neighbour is refined, in face order); -1 for none.
constexpr int FINE_WORD = 27;
constexpr int NT = 256;  // threads per CTA

template <int DIM>
struct BG {
  static constexpr int CB = DIM == 3 ? BS * BS * BS : BS * BS;       // cells per block
  static constexpr int WN = DIM == 3 ? PAD * PAD * PAD : PAD * PAD;  // primitive texels per slot
  static constexpr int PN = DIM == 3 ? PP * PP * PP : PP * PP;       // half-step texels per slot
};

__device__ __forceinline__ int bt_at(const int* __restrict__ bt, int slot, int i) { return __ldg(bt + slot * BTS + i); }
__device__ __forceinline__ bool leaf_of(const int* __restrict__ bt, int slot) { return (bt_at(bt, slot, 4) & 2) != 0; }

template <int DIM>
__device__ __forceinline__ int cell_ix(const int* l) {
  return DIM == 3 ? (l[2] * BS + l[1]) * BS + l[0] : l[1] * BS + l[0];
}
template <int DIM>
__device__ __forceinline__ int wtex(const int* l) {
  return DIM == 3 ? ((l[2] + NG) * PAD + (l[1] + NG)) * PAD + (l[0] + NG) : (l[1] + NG) * PAD + (l[0] + NG);
}
template <int DIM>
__device__ __forceinline__ int ptex(const int* l) {
  return DIM == 3 ? ((l[2] + 1) * PP + (l[1] + 1)) * PP + (l[0] + 1) : (l[1] + 1) * PP + (l[0] + 1);
}

// Where the value of a (possibly ghost) cell of a block comes from (amr/grid.wgsl:186-222):
// kind 0 a cell at the same level (the block's own, a neighbour's, or its image across a
// boundary of the domain, with velocity signs), kind 1 beyond a face whose neighbour is one
// level coarser (slot = that coarser leaf), kind 2 an edge or corner ghost.
struct Src {
  int kind, slot;
  int from;  // the block in whose frame l is given (kind 1: the fine block beside the coarse leaf)
  int l[3];
  float flip[3];
};

template <int DIM>
__device__ __forceinline__ Src ghost_src(const int* __restrict__ bt, int slot, const int* l) {
  Src s;
  s.kind = 0;
  s.slot = slot;
  s.from = slot;
  s.l[0] = l[0]; s.l[1] = l[1]; s.l[2] = l[2];
  s.flip[0] = s.flip[1] = s.flip[2] = 1.f;
  int out = 0, axis = 0;
#pragma unroll
  for (int a = 0; a < DIM; a++)
    if (l[a] < 0 || l[a] >= BS) { out++; axis = a; }
  if (out == 0) return s;
  if (out > 1) { s.kind = 2; return s; }
  const int upper = l[axis] >= BS ? 1 : 0;
  const int nb = bt_at(bt, slot, 6 + 2 * axis + upper);
  if (nb >= 0) {
    s.slot = nb;
    s.l[axis] = l[axis] + (upper ? -BS : BS);
  } else if (nb == -1) {
    s.kind = 1;
    s.slot = bt_at(bt, slot, 20 + 2 * axis + upper);
  } else {
    // a face of the domain of kind -1 - nb (hydro/boundary.wgsl:47-52): mirror image beyond a
    // wall, the edge cell beyond an outflow face
    const int k = -1 - nb;
    if (k == 2) {
      s.l[axis] = upper ? 2 * BS - 1 - l[axis] : -1 - l[axis];
      s.flip[axis] = -1.f;
    } else {
      s.l[axis] = upper ? BS - 1 : 0;
    }
  }
  return s;
}

// An edge or corner ghost, resolved one axis at a time: across the first out-of-range axis to
// the same-level neighbour (or the boundary image), then the rest in that block's own frame, so
// that it holds the value that the neighbour's own ghost there holds. That is what the
// reference's predictor sees when it predicts a face ghost at its source (amr/predict.wgsl:184),
// and hops in either order reach the same cell. Where a hop meets a coarser block before the last
// axis, the remaining axes are clamped into the block (the face ghost beside it): such a ghost is
// predicted in place with those axes' slopes masked. (The reference leaves edge ghosts unwritten,
// amr/assemble.wgsl:86; its masked rim ghosts then read whatever the texture held.)
template <int DIM>
__device__ __forceinline__ Src ghost_src_any(const int* __restrict__ bt, int slot, const int* l) {
  int cur = slot;
  int m[3] = {l[0], l[1], l[2]};
  float flip[3] = {1.f, 1.f, 1.f};
#pragma unroll
  for (int hop = 0; hop < DIM; hop++) {
    int out = 0, axis = -1;
#pragma unroll
    for (int a = 0; a < DIM; a++)
      if (m[a] < 0 || m[a] >= BS) {
        out++;
        if (axis < 0) axis = a;
      }
    if (out <= 1) break;
    const int upper = m[axis] >= BS ? 1 : 0;
    const int nb = bt_at(bt, cur, 6 + 2 * axis + upper);
    if (nb >= 0) {
      cur = nb;
      m[axis] += upper ? -BS : BS;
    } else if (nb <= -2) {
      if (-1 - nb == 2) {
        m[axis] = upper ? 2 * BS - 1 - m[axis] : -1 - m[axis];
        flip[axis] = -flip[axis];
      } else {
        m[axis] = upper ? BS - 1 : 0;
      }
    } else {
      // a coarser block across this axis: the face ghost beside the texel
#pragma unroll
      for (int a = 0; a < DIM; a++)
        if (a != axis) m[a] = min(max(m[a], 0), BS - 1);
    }
  }
  Src s = ghost_src<DIM>(bt, cur, m);
#pragma unroll
  for (int a = 0; a < 3; a++) s.flip[a] *= flip[a];
  return s;
}

struct Cons {
  float4 a, b;
};

// The conserved state of cell l of a same-level block (amr/cons.wgsl:19-43 u_at): a leaf's own
// cell, or the mean of the 2^ndim cells of the leaf child under it.
template <int DIM>
__device__ __forceinline__ Cons u_at(const int* __restrict__ bt, const float4* __restrict__ u1, const float4* __restrict__ u2,
                                     int slot, const int* lin) {
  // (the index is inside the block by construction; clamped so that no table can send a read
  // outside the atlas)
  const int l[3] = {min(max(lin[0], 0), BS - 1), min(max(lin[1], 0), BS - 1), DIM == 3 ? min(max(lin[2], 0), BS - 1) : 0};
  if (leaf_of(bt, slot)) {
    const size_t o = (size_t)slot * BG<DIM>::CB + cell_ix<DIM>(l);
    return Cons{__ldg(u1 + o), __ldg(u2 + o)};
  }
  int h[3] = {l[0] >= BS / 2, l[1] >= BS / 2, DIM == 3 ? (l[2] >= BS / 2) : 0};
  const int ch = bt_at(bt, slot, 12 + (h[0] | (h[1] << 1) | (h[2] << 2)));
  if (ch < 0 || !leaf_of(bt, ch)) return Cons{make_float4(1.f, 0.f, 0.f, 0.f), make_float4(1.f, 1.f, 0.f, 0.f)};
  float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
  const int nz = DIM == 3 ? 2 : 1;
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < 2; j++)
      for (int i = 0; i < 2; i++) {
        int f[3] = {2 * (l[0] - (BS / 2) * h[0]) + i, 2 * (l[1] - (BS / 2) * h[1]) + j,
                    DIM == 3 ? 2 * (l[2] - (BS / 2) * h[2]) + k : 0};
        const size_t o = (size_t)ch * BG<DIM>::CB + cell_ix<DIM>(f);
        const float4 x = __ldg(u1 + o), y = __ldg(u2 + o);
        a.x += x.x; a.y += x.y; a.z += x.z; a.w += x.w;
        b.x += y.x; b.y += y.y; b.z += y.z; b.w += y.w;
      }
  const float w = DIM == 3 ? 0.125f : 0.25f;
  return Cons{make_float4(a.x * w, a.y * w, a.z * w, a.w * w), make_float4(b.x * w, b.y * w, b.z * w, b.w * w)};
}

// amr/cons.wgsl u_near: the conserved state of a kind-0 cell near a coarse block, with the
// boundary's velocity signs.
template <int DIM>
__device__ __forceinline__ bool u_near(const int* __restrict__ bt, const float4* __restrict__ u1, const float4* __restrict__ u2,
                                       int slot, const int* l, Cons& u) {
  const Src s = ghost_src<DIM>(bt, slot, l);
  if (s.kind != 0) return false;
  u = u_at<DIM>(bt, u1, u2, s.slot, s.l);
  u.a.y *= s.flip[0];
  u.a.z *= s.flip[1];
  u.a.w *= s.flip[2];
  return true;
}

// The prolongation's single slope per component (the limiter's limit4: MC for Koren and MC,
// else the limiter itself; amr/cons.wgsl:53-66 slope_between with the product-rule momentum).
template <int R>
__device__ __forceinline__ float lim4(float a, float b) {
  return limit<R == R_KOREN ? R_MC : R>(a, b, 0.f);
}
template <int R>
__device__ __forceinline__ Cons slope_between(const Cons& c, const Cons& m, const Cons& p, float rho_floor) {
  Cons s;
  s.a.x = lim4<R>(c.a.x - m.a.x, p.a.x - c.a.x);
  const float ic = 1.f / fmaxf(c.a.x, rho_floor), im = 1.f / fmaxf(m.a.x, rho_floor), ip = 1.f / fmaxf(p.a.x, rho_floor);
  const float vc[3] = {c.a.y * ic, c.a.z * ic, c.a.w * ic};
  const float vm[3] = {m.a.y * im, m.a.z * im, m.a.w * im};
  const float vp[3] = {p.a.y * ip, p.a.z * ip, p.a.w * ip};
  float sm[3];
#pragma unroll
  for (int i = 0; i < 3; i++) sm[i] = vc[i] * s.a.x + c.a.x * lim4<R>(vc[i] - vm[i], vp[i] - vc[i]);
  s.a.y = sm[0]; s.a.z = sm[1]; s.a.w = sm[2];
  s.b.x = lim4<R>(c.b.x - m.b.x, p.b.x - c.b.x);
  s.b.y = lim4<R>(c.b.y - m.b.y, p.b.y - c.b.y);
  s.b.z = lim4<R>(c.b.z - m.b.z, p.b.z - c.b.z);
  s.b.w = lim4<R>(c.b.w - m.b.w, p.b.w - c.b.w);
  return s;
}

struct Slopes {
  Cons s[3];
  float f;
};

// amr/cons.wgsl:78-125 prolong_slopes / prolong_child: limited slopes scaled back by one common
// factor so that the children's density, energy and internal energy stay positive.
template <int DIM, int R>
__device__ __forceinline__ Slopes prolong_slopes(const Cons& uc, const Cons* m, const bool* mok, const Cons* p,
                                                 const bool* pok, float rho_floor) {
  Slopes sl;
  float drop[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int a = 0; a < 3; a++) {
    sl.s[a] = Cons{make_float4(0.f, 0.f, 0.f, 0.f), make_float4(0.f, 0.f, 0.f, 0.f)};
    if (a < DIM && mok[a] && pok[a]) sl.s[a] = slope_between<R>(uc, m[a], p[a], rho_floor);
    drop[0] += fabsf(sl.s[a].a.x);
    drop[1] += fabsf(sl.s[a].b.x);
    drop[2] += fabsf(sl.s[a].b.y);
  }
  const float room[3] = {0.5f * fmaxf(uc.a.x, 0.f), 0.5f * fmaxf(uc.b.x, 0.f), 0.5f * fmaxf(uc.b.y, 0.f)};
  float f = 1.f;
#pragma unroll
  for (int i = 0; i < 3; i++) f = fminf(f, fminf(1.f, room[i] / fmaxf(0.25f * drop[i], 1e-37f)));
  sl.f = f;
  return sl;
}
__device__ __forceinline__ Cons prolong_child(const Cons& uc, const Slopes& s, const int* par) {
  const float o0 = s.f * (par[0] - 0.5f) * 0.5f, o1 = s.f * (par[1] - 0.5f) * 0.5f, o2 = s.f * (par[2] - 0.5f) * 0.5f;
  Cons u;
  u.a.x = uc.a.x + o0 * s.s[0].a.x + o1 * s.s[1].a.x + o2 * s.s[2].a.x;
  u.a.y = uc.a.y + o0 * s.s[0].a.y + o1 * s.s[1].a.y + o2 * s.s[2].a.y;
  u.a.z = uc.a.z + o0 * s.s[0].a.z + o1 * s.s[1].a.z + o2 * s.s[2].a.z;
  u.a.w = uc.a.w + o0 * s.s[0].a.w + o1 * s.s[1].a.w + o2 * s.s[2].a.w;
  u.b.x = uc.b.x + o0 * s.s[0].b.x + o1 * s.s[1].b.x + o2 * s.s[2].b.x;
  u.b.y = uc.b.y + o0 * s.s[0].b.y + o1 * s.s[1].b.y + o2 * s.s[2].b.y;
  u.b.z = uc.b.z + o0 * s.s[0].b.z + o1 * s.s[1].b.z + o2 * s.s[2].b.z;
  u.b.w = uc.b.w + o0 * s.s[0].b.w + o1 * s.s[1].b.w + o2 * s.s[2].b.w;
  return u;
}

// The coarse cell under texel l of block `slot`, in the coarser leaf `cs`: its state and the
// prolongation's limited slopes (amr/assemble.wgsl:47-75, amr/cons.wgsl:78-106), and the texel's
// parity within it. Every fine texel over one coarse cell gets the same state and slopes.
template <int DIM, int R>
__device__ __forceinline__ void coarse_cell(const int* __restrict__ bt, const float4* __restrict__ u1,
                                            const float4* __restrict__ u2, int nr, int slot, const int* l, int cs,
                                            float rho_floor, Cons& uc, Slopes& sl, int* par) {
  const int nc = nr * BS << bt_at(bt, cs, 0);
  int gf[3], lc[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    gf[a] = a < DIM ? bt_at(bt, slot, 1 + a) * BS + l[a] : 0;
    int gc = gf[a] >> 1;
    gc = ((gc % nc) + nc) % nc;
    lc[a] = a < DIM ? gc - bt_at(bt, cs, 1 + a) * BS : 0;
    par[a] = a < DIM ? (gf[a] & 1) : 0;
  }
  Cons m[3], p[3];
  bool mok[3] = {false, false, false}, pok[3] = {false, false, false};
  if (!u_near<DIM>(bt, u1, u2, cs, lc, uc)) uc = Cons{make_float4(1.f, 0.f, 0.f, 0.f), make_float4(1.f, 1.f, 0.f, 0.f)};
#pragma unroll
  for (int a = 0; a < DIM; a++) {
    int at[3] = {lc[0], lc[1], lc[2]};
    at[a] -= 1;
    mok[a] = u_near<DIM>(bt, u1, u2, cs, at, m[a]);
    at[a] += 2;
    pok[a] = u_near<DIM>(bt, u1, u2, cs, at, p[a]);
  }
  sl = prolong_slopes<DIM, R>(uc, m, mok, p, pok, rho_floor);
}

// amr/assemble.wgsl:47-75 from_coarse: a ghost beyond a face whose neighbour is one level
// coarser, prolonged from the coarse leaf `cs` with slopes from that leaf's neighbours.
template <int DIM, int R>
__device__ __forceinline__ Cons from_coarse(const int* __restrict__ bt, const float4* __restrict__ u1,
                                            const float4* __restrict__ u2, int nr, int slot, const int* l, int cs,
                                            float rho_floor) {  // nr: root blocks per side of the block's grid
  Cons uc;
  Slopes sl;
  int par[3];
  coarse_cell<DIM, R>(bt, u1, u2, nr, slot, l, cs, rho_floor, uc, sl, par);
  return prolong_child(uc, sl, par);
}

__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float block_max(float v, float* sRed) {
  v = warp_max_f(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sRed[warp] = v;
  __syncthreads();
  float m = lane < NT / 32 ? sRed[lane] : 0.f;
  return warp_max_f(m);
}
__device__ __forceinline__ float rate_guard_f(float r) { return (r == r) ? r : __int_as_float(0x7f800000); }

template <int DIM>
__device__ __forceinline__ void load_w(const float4* __restrict__ w1, const float4* __restrict__ w2, int slot, const int* l,
                                       float* w) {
  const size_t o = (size_t)slot * BG<DIM>::WN + wtex<DIM>(l);
  const float4 a = __ldg(w1 + o), b = __ldg(w2 + o);
  w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
  w[4] = b.x; w[5] = b.y; w[6] = b.z;
}

// Per-block timesteps (amr/bins_on.wgsl). Time advances in cycles of 2^K substeps of the fastest
// block's step; a block in bin k steps 2^k substeps at a time, starting on substeps that are
// multiples of 2^k. The bin table holds [0] the substep being taken and [1 + slot] each block's
// bin; a null table is one timestep for every block (amr/bins_off.wgsl).
__device__ __forceinline__ int blk_bin(const int* __restrict__ bins, int slot) {
  return bins ? __ldg(bins + 1 + slot) : 0;
}
// The block starts a step on this substep.
__device__ __forceinline__ bool blk_active(const int* __restrict__ bins, int slot) {
  if (!bins) return true;
  return (__ldg(bins) & ((1 << __ldg(bins + 1 + slot)) - 1)) == 0;
}
// A leaf part way through a longer step (amr/mid_on.wgsl mid_block): its stored state is already
// that of the end of its step, and its neighbours take its half-step prediction instead.
__device__ __forceinline__ bool mid_block(const int* __restrict__ bt, const int* __restrict__ bins, int slot) {
  return bins && leaf_of(bt, slot) && !blk_active(bins, slot);
}
// The conserved state at cell l (interior or first ghost layer) of block `slot` at the middle of
// its step, from the half-step atlas its prediction wrote when the step began
// (amr/mid_on.wgsl:18-31 mid_cons; ideal gas, e = p / (gamma - 1)).
template <int DIM>
__device__ __forceinline__ Cons mid_cons(const KParams& P, const float4* __restrict__ p1, const float4* __restrict__ p2,
                                         int slot, const int* l) {
  const size_t o = (size_t)slot * BG<DIM>::PN + ptex<DIM>(l);
  const float4 a = __ldg(p1 + o), b = __ldg(p2 + o);
  const float rho = a.x;
  const float eint = b.x * P.inv_gm1;
  return Cons{make_float4(rho, rho * a.y, rho * a.z, rho * a.w),
              make_float4(eint + 0.5f * rho * (a.y * a.y + a.z * a.z + a.w * a.w), eint, rho * b.y, 0.f)};
}

// coarse_cell for a coarse leaf part way through its step: the coarse cell and its neighbours
// along the axes from its half-step atlas (which covers its first ghost layer, so no boundary
// mapping is needed; amr/assemble.wgsl:59-66).
template <int DIM, int R>
__device__ __forceinline__ void coarse_cell_mid(const KParams& P, const int* __restrict__ bt, const float4* __restrict__ p1,
                                                const float4* __restrict__ p2, int nr, int slot, const int* l, int cs,
                                                Cons& uc, Slopes& sl, int* par) {
  const int nc = nr * BS << bt_at(bt, cs, 0);
  int lc[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int gf = a < DIM ? bt_at(bt, slot, 1 + a) * BS + l[a] : 0;
    int gc = gf >> 1;
    gc = ((gc % nc) + nc) % nc;
    lc[a] = a < DIM ? gc - bt_at(bt, cs, 1 + a) * BS : 0;
    par[a] = a < DIM ? (gf & 1) : 0;
  }
  uc = mid_cons<DIM>(P, p1, p2, cs, lc);
  Cons m[3], p[3];
  bool ok[3] = {true, true, true};
#pragma unroll
  for (int a = 0; a < DIM; a++) {
    int at[3] = {lc[0], lc[1], lc[2]};
    at[a] -= 1;
    m[a] = mid_cons<DIM>(P, p1, p2, cs, at);
    at[a] += 2;
    p[a] = mid_cons<DIM>(P, p1, p2, cs, at);
  }
  sl = prolong_slopes<DIM, R>(uc, m, ok, p, ok, P.rho_floor);
}
template <int DIM, int R>
__device__ __forceinline__ Cons from_coarse_mid(const KParams& P, const int* __restrict__ bt, const float4* __restrict__ p1,
                                                const float4* __restrict__ p2, int nr, int slot, const int* l, int cs) {
  Cons uc;
  Slopes sl;
  int par[3];
  coarse_cell_mid<DIM, R>(P, bt, p1, p2, nr, slot, l, cs, uc, sl, par);
  return prolong_child(uc, sl, par);
}

}  // namespace amrk

// Persistent work-list grids: `per_sm` CTAs on each of the 148 SMs, or one per block when fewer.
inline int grid_for(int n, int per_sm) {
  int g = 148 * per_sm;
  if (n < g) g = n;
  return g < 1 ? 1 : g;
}

#define SHZ_RECON_SWITCH(recon, ISEN, CALL)                                  \
  switch (recon) {                                                           \
    case R_MINMOD: { constexpr int R = R_MINMOD; CALL; break; }             \
    case R_MC: { constexpr int R = R_MC; CALL; break; }                     \
    case R_VANLEER: { constexpr int R = R_VANLEER; CALL; break; }           \
    default: { constexpr int R = R_KOREN; CALL; break; }                    \
  }

}  // namespace shz
