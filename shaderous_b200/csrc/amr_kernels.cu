// The passes of one step on the adaptive block grid, as persistent work-list kernels.
//
// A block holds 16^ndim cells. Three atlases live in HBM, slot-major, with x fastest:
//   - the conserved state: two parities of 16^ndim cells x (u1, u2) float4;
//   - the primitives with two ghost layers: 20^ndim cells x (w1 = rho, v; w2 = p, s, cs, 0);
//   - the half-step states over the block and one ghost layer: 18^ndim cells x
//     (p1 = rho, v; p2 = p, s, shock flag, first-order flag).
// One step is three or four kernels, captured in a CUDA graph by the host:
//   1. amr_assemble over every block (leaves and parents): primitives with ghost fill.
//   2. clock_multi_kernel: dt.
//   3. amr_fine_flux over the faces whose same-level neighbour is refined: the mean fine fluxes
//      (only when the mesh has such faces).
//   4. amr_sweep over the leaves: half steps, fluxes and the update, in one pass over the
//      primitives, the matched faces' fluxes read from the buffer step 3 filled.
// The reference's own pass structure is kept beside it as a cross-check (two_pass): amr_predict
// writes the half steps to their atlas and amr_update reads them.
// This follows the reference's AmrSim.encodeSteps (src/amr/amr_sim.ts:2709-2946), and its rules
// for the ghost fill (amr/grid.wgsl:186-222 ghost_src; amr/cons.wgsl:19-125 restriction and
// prolongation; amr/assemble.wgsl:47-75 from_coarse), the predictor at the source
// (amr/predict.wgsl:184-221) and the matching of coarse faces to the mean of the fine fluxes
// (amr/update.wgsl:207-295). Every kernel walks a device list of block slots with a fixed grid of
// CTAs, one block at a time per CTA.
#include <cuda_runtime.h>
#include <algorithm>
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

// amr/assemble.wgsl:47-75 from_coarse: a ghost beyond a face whose neighbour is one level
// coarser, prolonged from the coarse leaf `cs` with slopes from that leaf's neighbours.
template <int DIM, int R>
__device__ __forceinline__ Cons from_coarse(const int* __restrict__ bt, const float4* __restrict__ u1,
                                            const float4* __restrict__ u2, int nr, int slot, const int* l, int cs,
                                            float rho_floor) {  // nr: root blocks per side of the block's grid
  const int nc = nr * BS << bt_at(bt, cs, 0);
  int gf[3], lc[3], par[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    gf[a] = a < DIM ? bt_at(bt, slot, 1 + a) * BS + l[a] : 0;
    int gc = gf[a] >> 1;
    gc = ((gc % nc) + nc) % nc;
    lc[a] = a < DIM ? gc - bt_at(bt, cs, 1 + a) * BS : 0;
    par[a] = a < DIM ? (gf[a] & 1) : 0;
  }
  Cons uc, m[3], p[3];
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
  const Slopes sl = prolong_slopes<DIM, R>(uc, m, mok, p, pok, rho_floor);
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

// 1. Primitives of every block in the list with two ghost layers; the rate / dx maximum over the
// leaves' own cells (assemble.wgsl:78-154; PER_DX in clock.wgsl).
template <int DIM, int R>
__global__ void __launch_bounds__(NT) amr_assemble(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                   const int* __restrict__ list, int n, const float4* __restrict__ u1,
                                                   const float4* __restrict__ u2, float4* __restrict__ w1,
                                                   float4* __restrict__ w2, unsigned* __restrict__ rates, int rslot) {
  __shared__ float sRed[NT / 32];
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    float rmax = 0.f;
    const int slot = __ldg(list + i);
    const int g = bt_at(bt, slot, GRID_WORD);
    const KParams& P = gp[g];
    const int nr = P.n[0];
    const bool leaf = leaf_of(bt, slot);
    const float inv_dx = (float)(ldexp(1.0, bt_at(bt, slot, 0)) / P.dx);
    for (int t = threadIdx.x; t < BG<DIM>::WN; t += NT) {
      int l[3] = {t % PAD - NG, (t / PAD) % PAD - NG, DIM == 3 ? t / (PAD * PAD) - NG : 0};
      const Src s = ghost_src_any<DIM>(bt, slot, l);
      Cons u;
      if (s.kind == 0) {
        u = u_at<DIM>(bt, u1, u2, s.slot, s.l);
        u.a.y *= s.flip[0];
        u.a.z *= s.flip[1];
        u.a.w *= s.flip[2];
      } else {
        u = from_coarse<DIM, R>(bt, u1, u2, nr, s.from, s.l, s.slot, P.rho_floor);
        u.a.y *= s.flip[0];
        u.a.z *= s.flip[1];
        u.a.w *= s.flip[2];
      }
      float w[7];
      prim_from_cons(u.a, u.b, P, 1.f, 1.f, 1.f, w);
      const size_t o = (size_t)slot * BG<DIM>::WN + t;
      w1[o] = make_float4(w[0], w[1], w[2], w[3]);
      w2[o] = make_float4(w[4], w[5], w[6], 0.f);
      bool inside = leaf;
#pragma unroll
      for (int a = 0; a < DIM; a++) inside = inside && l[a] >= 0 && l[a] < BS;
      if (inside) rmax = fmaxf(rmax, rate_guard_f(fabsf(w[1]) + fabsf(w[2]) + fabsf(w[3]) + P.signal * w[6]) * inv_dx);
    }
    const float m = block_max(rmax, sRed);
    if (threadIdx.x == 0 && leaf) atomicMax(rates + 2 * g + rslot, __float_as_uint(m));
  }
}

template <int DIM>
__device__ __forceinline__ void load_w(const float4* __restrict__ w1, const float4* __restrict__ w2, int slot, const int* l,
                                       float* w) {
  const size_t o = (size_t)slot * BG<DIM>::WN + wtex<DIM>(l);
  const float4 a = __ldg(w1 + o), b = __ldg(w2 + o);
  w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
  w[4] = b.x; w[5] = b.y; w[6] = b.z;
}

// 2. Half steps of every leaf over its cells and first ghost layer (predict.wgsl:184-221): a
// same-level or boundary ghost is predicted at its source and mirrored; a ghost beside a coarser
// block in place, its transverse slopes dropped at the rim of the face.
template <int DIM, int R, bool ISEN>
__global__ void __launch_bounds__(NT) amr_predict(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                  const int* __restrict__ list, int n, const float4* __restrict__ w1,
                                                  const float4* __restrict__ w2, float4* __restrict__ p1,
                                                  float4* __restrict__ p2, const DevClock* __restrict__ clks) {
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int slot = __ldg(list + i);
    const int g = bt_at(bt, slot, GRID_WORD);
    const KParams& P = gp[g];
    const double dt = clks[g].dt;
    const float h = (float)((0.5 * dt) * ldexp(1.0, bt_at(bt, slot, 0)) / P.dx);
    for (int t = threadIdx.x; t < BG<DIM>::PN; t += NT) {
      int l[3] = {t % PP - 1, (t / PP) % PP - 1, DIM == 3 ? t / (PP * PP) - 1 : 0};
      const Src s = ghost_src<DIM>(bt, slot, l);
      if (s.kind == 2) continue;
      const bool at_source = s.kind == 0;
      const int src = at_source ? s.slot : slot;
      int c0[3] = {at_source ? s.l[0] : l[0], at_source ? s.l[1] : l[1], at_source ? s.l[2] : l[2]};
      float mask[3] = {1.f, 1.f, 1.f};
      if (!at_source)
#pragma unroll
        for (int a = 0; a < DIM; a++) mask[a] = (l[a] == 0 || l[a] == BS - 1) ? 0.f : 1.f;
      float c[7];
      load_w<DIM>(w1, w2, src, c0, c);
      float su[DIM][6], sd[DIM][6];
      float conv = 0.f, jump = 0.f;
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
        jump = fmaxf(jump, fabsf(p[4] - m[4]) / fminf(p[4], m[4]));
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
// the 2^(ndim-1) fine faces it covers, computed as the fine leaf computes them.
template <int DIM, int R, bool ISEN, int AXIS>
__device__ __forceinline__ void match_face(const KParams& P, const int* __restrict__ bt, const float4* __restrict__ w1,
                                           const float4* __restrict__ w2, const float4* __restrict__ p1,
                                           const float4* __restrict__ p2, int slot, const int* l, bool hi, float* F) {
  const int np = bt_at(bt, slot, 6 + 2 * AXIS + (hi ? 1 : 0));
  if (np < 0 || leaf_of(bt, np)) return;
  const bool upper = !hi;
  int h[3] = {l[0] >= BS / 2, l[1] >= BS / 2, DIM == 3 ? (l[2] >= BS / 2) : 0};
  int bits[3] = {h[0], h[1], h[2]};
  bits[AXIS] = upper ? 1 : 0;
  if (DIM == 2) bits[2] = 0;
  const int ch = bt_at(bt, np, 12 + (bits[0] | (bits[1] << 1) | (bits[2] << 2)));
  if (ch < 0) return;
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
  const float w = 1.f / (float)(n1 * n2);
#pragma unroll
  for (int v = 0; v < 8; v++) F[v] = sum[v] * w;
}

// 3. Fluxes and the update of every leaf (update.wgsl:327-560). A CTA takes a block plane by
// plane along z; each thread owns a column and solves its lower x and y faces (the last row
// also the block's upper face) into shared memory, and its z faces in registers, so every face
// is solved once.
template <int DIM, int R, bool ISEN>
__global__ void __launch_bounds__(NT) amr_update(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                 const int* __restrict__ list, int n, const float4* __restrict__ u1,
                                                 const float4* __restrict__ u2, const float4* __restrict__ w1,
                                                 const float4* __restrict__ w2, const float4* __restrict__ p1,
                                                 const float4* __restrict__ p2, float4* __restrict__ o1,
                                                 float4* __restrict__ o2, const DevClock* __restrict__ clks) {
  __shared__ float sFx[8][BS * (BS + 1)];
  __shared__ float sFy[8][BS * (BS + 1)];
  const int tx = threadIdx.x % BS, ty = threadIdx.x / BS;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int slot = __ldg(list + i);
    const int g = bt_at(bt, slot, GRID_WORD);
    const KParams& P = gp[g];
    const double dt = clks[g].dt;
    const bool held = clks[g].held != 0;
    const float dtdx = (float)(dt * ldexp(1.0, bt_at(bt, slot, 0)) / P.dx);
    float Fzlo[8];
    const int nk = DIM == 3 ? BS : 1;
    for (int k = 0; k < nk; k++) {
      int l[3] = {tx, ty, k};
      float F[8];
      // x faces
      {
        int a[3] = {tx - 1, ty, k};
        face_flux<DIM, R, ISEN, 0>(P, w1, w2, p1, p2, slot, a, F);
        if (tx == 0) match_face<DIM, R, ISEN, 0>(P, bt, w1, w2, p1, p2, slot, l, false, F);
#pragma unroll
        for (int v = 0; v < 8; v++) sFx[v][ty * (BS + 1) + tx] = F[v];
        if (tx == BS - 1) {
          face_flux<DIM, R, ISEN, 0>(P, w1, w2, p1, p2, slot, l, F);
          match_face<DIM, R, ISEN, 0>(P, bt, w1, w2, p1, p2, slot, l, true, F);
#pragma unroll
          for (int v = 0; v < 8; v++) sFx[v][ty * (BS + 1) + BS] = F[v];
        }
      }
      // y faces
      {
        int a[3] = {tx, ty - 1, k};
        face_flux<DIM, R, ISEN, 1>(P, w1, w2, p1, p2, slot, a, F);
        if (ty == 0) match_face<DIM, R, ISEN, 1>(P, bt, w1, w2, p1, p2, slot, l, false, F);
#pragma unroll
        for (int v = 0; v < 8; v++) sFy[v][ty * BS + tx] = F[v];
        if (ty == BS - 1) {
          face_flux<DIM, R, ISEN, 1>(P, w1, w2, p1, p2, slot, l, F);
          match_face<DIM, R, ISEN, 1>(P, bt, w1, w2, p1, p2, slot, l, true, F);
#pragma unroll
          for (int v = 0; v < 8; v++) sFy[v][BS * BS + tx] = F[v];
        }
      }
      float Fzhi[8];
      if constexpr (DIM == 3) {
        if (k == 0) {
          int a[3] = {tx, ty, -1};
          face_flux<DIM, R, ISEN, 2>(P, w1, w2, p1, p2, slot, a, Fzlo);
          match_face<DIM, R, ISEN, 2>(P, bt, w1, w2, p1, p2, slot, l, false, Fzlo);
        }
        face_flux<DIM, R, ISEN, 2>(P, w1, w2, p1, p2, slot, l, Fzhi);
        if (k == BS - 1) match_face<DIM, R, ISEN, 2>(P, bt, w1, w2, p1, p2, slot, l, true, Fzhi);
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
      const float4 a = __ldg(u1 + oc), b = __ldg(u2 + oc);
      if (held) {
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

// Löhner's refinement indicator per leaf (amr/flag.wgsl:66-155): the largest over the block's
// cells of the normalised second differences of density and pressure (EPS = 0.01), at least
// GAS_MIN.
template <int DIM>
__global__ void __launch_bounds__(NT) amr_flag(const int* __restrict__ list, int n, const float4* __restrict__ w1,
                                               const float4* __restrict__ w2, float* __restrict__ flags) {
  __shared__ float sRed[NT / 32];
  const float EPS = 0.01f;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int slot = __ldg(list + i);
    float m = 0.f;
    for (int t = threadIdx.x; t < BG<DIM>::CB; t += NT) {
      int l[3] = {t % BS, (t / BS) % BS, DIM == 3 ? t / (BS * BS) : 0};
      const size_t o = (size_t)slot * BG<DIM>::WN + wtex<DIM>(l);
      const float r0 = __ldg(w1 + o).x, p0 = __ldg(w2 + o).x;
      float nr = 0.f, dr = 0.f, np = 0.f, dp = 0.f;
#pragma unroll
      for (int a = 0; a < DIM; a++) {
        int lp[3] = {l[0], l[1], l[2]}, lm[3] = {l[0], l[1], l[2]};
        lp[a] += 1;
        lm[a] -= 1;
        const size_t op = (size_t)slot * BG<DIM>::WN + wtex<DIM>(lp), om = (size_t)slot * BG<DIM>::WN + wtex<DIM>(lm);
        const float rp = __ldg(w1 + op).x, rm = __ldg(w1 + om).x, pp = __ldg(w2 + op).x, pm = __ldg(w2 + om).x;
        const float sr = rp - 2.f * r0 + rm, sp = pp - 2.f * p0 + pm;
        const float er = fabsf(rp - r0) + fabsf(r0 - rm) + EPS * (fabsf(rp) + 2.f * fabsf(r0) + fabsf(rm));
        const float ep = fabsf(pp - p0) + fabsf(p0 - pm) + EPS * (fabsf(pp) + 2.f * fabsf(p0) + fabsf(pm));
        nr += sr * sr;
        dr += er * er;
        np += sp * sp;
        dp += ep * ep;
      }
      const float ind = fmaxf(sqrtf(nr / fmaxf(dr, 1e-30f)), sqrtf(np / fmaxf(dp, 1e-30f)));
      m = fmaxf(m, ind);
    }
    m = block_max(m, sRed);
    if (threadIdx.x == 0) flags[slot] = fmaxf(m, 1e-30f);
  }
}

// Filling the leaves of a new tree from the old one (amr/regrid.wgsl:41-139): copy, restrict
// the eight old children, or prolong from the old leaf with the kinetic energy kept
// consistent (each child's own kinetic energy plus its interpolated internal energy, less one
// shared offset that keeps the mean total energy the coarse cell's).
template <int DIM, int R>
__global__ void __launch_bounds__(NT) amr_regrid(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                 const int* __restrict__ rg, const int* __restrict__ list,
                                                 int n, const float4* __restrict__ u1, const float4* __restrict__ u2,
                                                 const float4* __restrict__ w1, const float4* __restrict__ w2,
                                                 float4* __restrict__ o1, float4* __restrict__ o2) {
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int slot = __ldg(list + i);
    const KParams& P = gp[bt_at(bt, slot, GRID_WORD)];
    const int kind = __ldg(rg + slot * RGS), src = __ldg(rg + slot * RGS + 1), oct = __ldg(rg + slot * RGS + 2);
    for (int t = threadIdx.x; t < BG<DIM>::CB; t += NT) {
      int l[3] = {t % BS, (t / BS) % BS, DIM == 3 ? t / (BS * BS) : 0};
      Cons u;
      if (kind == 2) {
        int lc[3] = {(l[0] >> 1) + (BS / 2) * (oct & 1), (l[1] >> 1) + (BS / 2) * ((oct >> 1) & 1),
                     DIM == 3 ? (l[2] >> 1) + (BS / 2) * ((oct >> 2) & 1) : 0};
        const size_t oc = (size_t)src * BG<DIM>::CB + cell_ix<DIM>(lc);
        const Cons uc{__ldg(u1 + oc), __ldg(u2 + oc)};
        Cons m[3], p[3];
        bool ok[3] = {true, true, true};
#pragma unroll
        for (int a = 0; a < DIM; a++) {
          for (int sgn = -1; sgn <= 1; sgn += 2) {
            int at[3] = {lc[0], lc[1], lc[2]};
            at[a] += sgn;
            const size_t ow = (size_t)src * BG<DIM>::WN + wtex<DIM>(at);
            const float4 x = __ldg(w1 + ow), y = __ldg(w2 + ow);
            const float eint = y.x * P.inv_gm1;
            Cons c;
            c.a = make_float4(x.x, x.x * x.y, x.x * x.z, x.x * x.w);
            c.b = make_float4(eint + 0.5f * x.x * (x.y * x.y + x.z * x.z + x.w * x.w), eint, x.x * y.y, 0.f);
            (sgn < 0 ? m[a] : p[a]) = c;
          }
        }
        const Slopes sl = prolong_slopes<DIM, R>(uc, m, ok, p, ok, P.rho_floor);
        int par[3] = {l[0] & 1, l[1] & 1, DIM == 3 ? (l[2] & 1) : 0};
        u = prolong_child(uc, sl, par);
        float ke = 0.f;
        for (int kz = 0; kz < (DIM == 3 ? 2 : 1); kz++)
          for (int jy = 0; jy < 2; jy++)
            for (int ix = 0; ix < 2; ix++) {
              int pc[3] = {ix, jy, kz};
              const Cons c = prolong_child(uc, sl, pc);
              ke += 0.5f * (c.a.y * c.a.y + c.a.z * c.a.z + c.a.w * c.a.w) / fmaxf(c.a.x, P.rho_floor);
            }
        ke *= DIM == 3 ? 0.125f : 0.25f;
        u.b.x = 0.5f * (u.a.y * u.a.y + u.a.z * u.a.z + u.a.w * u.a.w) / fmaxf(u.a.x, P.rho_floor) + u.b.y +
                (uc.b.x - uc.b.y - ke);
      } else if (kind == 3) {
        int h[3] = {l[0] >= BS / 2, l[1] >= BS / 2, DIM == 3 ? (l[2] >= BS / 2) : 0};
        const int ch = __ldg(rg + slot * RGS + 4 + (h[0] | (h[1] << 1) | (h[2] << 2)));
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
        for (int kz = 0; kz < (DIM == 3 ? 2 : 1); kz++)
          for (int jy = 0; jy < 2; jy++)
            for (int ix = 0; ix < 2; ix++) {
              int f[3] = {2 * (l[0] - (BS / 2) * h[0]) + ix, 2 * (l[1] - (BS / 2) * h[1]) + jy,
                          DIM == 3 ? 2 * (l[2] - (BS / 2) * h[2]) + kz : 0};
              const size_t o = (size_t)ch * BG<DIM>::CB + cell_ix<DIM>(f);
              const float4 x = __ldg(u1 + o), y = __ldg(u2 + o);
              a.x += x.x; a.y += x.y; a.z += x.z; a.w += x.w;
              b.x += y.x; b.y += y.y; b.z += y.z; b.w += y.w;
            }
        const float w = DIM == 3 ? 0.125f : 0.25f;
        u.a = make_float4(a.x * w, a.y * w, a.z * w, a.w * w);
        u.b = make_float4(b.x * w, b.y * w, b.z * w, b.w * w);
      } else {
        const size_t o = (size_t)src * BG<DIM>::CB + t;
        u = Cons{__ldg(u1 + o), __ldg(u2 + o)};
      }
      const size_t o = (size_t)slot * BG<DIM>::CB + t;
      o1[o] = u.a;
      o2[o] = u.b;
    }
  }
}

// Conservation totals over the leaves in compensated float64, one partial row per CTA.
struct AccD {
  double s, c;
  __device__ void add(double x) {
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
};
template <int DIM>
__global__ void __launch_bounds__(NT) amr_diag(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                               const int* __restrict__ list, int n, const float4* __restrict__ u1,
                                               const float4* __restrict__ u2, double* __restrict__ part) {
  AccD acc[8];
  for (int i = 0; i < 8; i++) acc[i] = AccD{0.0, 0.0};
  double mach = 0.0;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int slot = __ldg(list + i);
    const KParams& P = gp[bt_at(bt, slot, GRID_WORD)];
    const double dx = P.dx / ldexp(1.0, bt_at(bt, slot, 0));
    const double dv = DIM == 3 ? dx * dx * dx : dx * dx;
    for (int t = threadIdx.x; t < BG<DIM>::CB; t += NT) {
      const size_t o = (size_t)slot * BG<DIM>::CB + t;
      const float4 a = __ldg(u1 + o), b = __ldg(u2 + o);
      const double rho = fmax((double)a.x, (double)P.rho_floor);
      const double vx = a.y / rho, vy = a.z / rho, vz = a.w / rho, v2 = vx * vx + vy * vy + vz * vz;
      const double p = fmax((double)P.gm1 * b.y, (double)P.p_floor);
      acc[0].add(rho * dv);
      acc[1].add((double)a.y * dv);
      acc[2].add((double)a.z * dv);
      acc[3].add((double)a.w * dv);
      acc[4].add(0.5 * rho * v2 * dv);
      acc[5].add(((double)b.x - 0.5 * rho * v2) * dv);
      acc[6].add((double)b.x * dv);
      acc[7].add((a.x <= P.rho_floor * 1.0001f || p <= P.p_floor * 1.0001) ? 1.0 : 0.0);
      mach = fmax(mach, sqrt(v2) / sqrt((double)P.gamma * p / rho));
    }
  }
  __shared__ double sh[NT][9];
  for (int v = 0; v < 8; v++) sh[threadIdx.x][v] = acc[v].s + acc[v].c;
  sh[threadIdx.x][8] = mach;
  __syncthreads();
  if (threadIdx.x < 9) {
    const int v = threadIdx.x;
    AccD s{0.0, 0.0};
    double mx = 0.0;
    for (int t = 0; t < NT; t++) {
      if (v == 8) mx = fmax(mx, sh[t][8]);
      else s.add(sh[t][v]);
    }
    part[(size_t)blockIdx.x * 9 + v] = v == 8 ? mx : s.s + s.c;
  }
}

__global__ void amr_diag_final(const double* __restrict__ part, int nblocks, double* __restrict__ out) {
  const int v = threadIdx.x;
  if (v >= 9) return;
  AccD s{0.0, 0.0};
  double mx = 0.0;
  for (int b = 0; b < nblocks; b++) {
    if (v == 8) mx = fmax(mx, part[(size_t)b * 9 + 8]);
    else s.add(part[(size_t)b * 9 + v]);
  }
  out[v] = v == 8 ? mx : s.s + s.c;
}

// The ghost classification of every texel of a block's primitive region, for checking the
// device's ghost indexing against the tables: (kind, slot, l0, l1, l2) per texel.
template <int DIM>
__global__ void amr_ghost_map(const int* __restrict__ bt, int slot, int* __restrict__ out) {
  for (int t = threadIdx.x + blockIdx.x * blockDim.x; t < BG<DIM>::WN; t += blockDim.x * gridDim.x) {
    int l[3] = {t % PAD - NG, (t / PAD) % PAD - NG, DIM == 3 ? t / (PAD * PAD) - NG : 0};
    const Src s = ghost_src<DIM>(bt, slot, l);
    out[t * 5 + 0] = s.kind;
    out[t * 5 + 1] = s.slot;
    out[t * 5 + 2] = s.l[0];
    out[t * 5 + 3] = s.l[1];
    out[t * 5 + 4] = s.l[2];
  }
}

// ---------------------------------------------------------------------------------------------
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

__device__ __forceinline__ void read_w6(const float* __restrict__ plane, int x, int y, float* w) {
#pragma unroll
  for (int c = 0; c < 6; c++) w[c] = plane[c * SWN + (y + NG) * PAD + (x + NG)];
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
template <int DIM, int R, bool ISEN>
__device__ __forceinline__ void predict_texel(const KParams& P, const int* __restrict__ bt, const float4* __restrict__ w1,
                                              const float4* __restrict__ w2, int slot, const int* l0, float h, int axis,
                                              Pred& pr, float* su, float* sd) {
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
    if (nb == -1) {
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
  float conv = 0.f, jump = 0.f;
  load_w6<DIM>(w1, w2, slot, l, c);
  with_cs(c, P);
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
    jump = fmaxf(jump, fabsf(p[4] - m[4]) / fminf(p[4], m[4]));
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
    load_w6<DIM>(w1, w2, slot, l0, g);
    with_cs(g, P);
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
template <int DIM, int R, bool ISEN, int AXIS>
__device__ __forceinline__ Flux8 fine_mean_flux(const KParams* __restrict__ Pp, const int* __restrict__ bt,
                                             const float4* __restrict__ w1, const float4* __restrict__ w2, int np, int l0,
                                             int l1, int l2, bool hi, float hf) {
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
      predict_texel<DIM, R, ISEN>(P, bt, w1, w2, ch, a, hf, AXIS, pa, sua, sda);
      predict_texel<DIM, R, ISEN>(P, bt, w1, w2, ch, b, hf, AXIS, pb, sub, sdb);
      float L[7], Rr[7], f[8];
      face_state(pa, sua, 1.f, L);
      face_state(pb, sdb, -1.f, Rr);
      riemann<AXIS>(L, Rr, P, f);
#pragma unroll
      for (int v = 0; v < 8; v++) out.v[v] += f[v];
    }
  const float w = 1.f / (float)(n1 * n2);
#pragma unroll
  for (int v = 0; v < 8; v++) out.v[v] *= w;
  return out;
}

// Fine-flux matching, ahead of the sweep (amr/update.wgsl:207-295): for every face of a leaf
// whose same-level neighbour is refined, the mean of the fine fluxes through each of its cells,
// into the buffer entry the host assigned (entries: leaf slot, face, index). One thread per face
// cell, so that the few blocks with such faces do not hold up a sweep's CTA.
template <int DIM, int R, bool ISEN>
__global__ void __launch_bounds__(NT) amr_fine_flux(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                    const int* __restrict__ flist, int nf, const float4* __restrict__ w1,
                                                    const float4* __restrict__ w2, const DevClock* __restrict__ clks,
                                                    float4* __restrict__ fbuf) {
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
    if (axis == 0) F = fine_mean_flux<DIM, R, ISEN, 0>(Pp, bt, w1, w2, np, edge, t1, t2, hi, hf);
    else if (axis == 1) F = fine_mean_flux<DIM, R, ISEN, 1>(Pp, bt, w1, w2, np, t1, edge, t2, hi, hf);
    else F = fine_mean_flux<DIM, R, ISEN, 2>(Pp, bt, w1, w2, np, t1, t2, edge, hi, hf);
    float4* o = fbuf + ((size_t)k * FC + c) * 2;
    o[0] = make_float4(F.v[0], F.v[1], F.v[2], F.v[3]);
    o[1] = make_float4(F.v[4], F.v[5], F.v[6], F.v[7]);
  }
}

// Shared memory of the block sweep, in floats.
constexpr int SW_RING = 3 * 6 * SWN;  // three planes of primitives
constexpr int SW_FACE = 2 * 7 * SPN;  // x and y upper face states of a plane
constexpr int SW_FLUX = 2 * 8 * SPN;  // x and y lower-face fluxes of a plane (also the half-step exchange)
constexpr int SW_KEEP = 8 * SPN;      // z boundary ghosts: a plane's half steps or the ghost's increments
constexpr size_t SWEEP_SMEM = (size_t)(SW_RING + SW_FACE + SW_FLUX + SW_KEEP) * sizeof(float);

template <int DIM, int R, bool ISEN>
__global__ void __maxnreg__(80)
    amr_sweep(const KParams* __restrict__ gp, const int* __restrict__ bt, const int* __restrict__ list, int n,
              const float4* __restrict__ u1, const float4* __restrict__ u2, const float4* __restrict__ w1,
              const float4* __restrict__ w2, float4* __restrict__ o1, float4* __restrict__ o2,
              const DevClock* __restrict__ clks, const float4* __restrict__ fbuf) {
  constexpr int FC = DIM == 3 ? BS * BS : BS;  // cells of a face
  extern __shared__ __align__(16) float smem[];
  float* sW = smem;
  float* sFace = sW + SW_RING;
  float* sFlux = sFace + SW_FACE;
  float* sKeep = sFlux + SW_FLUX;
  // the block's grid parameters, copied once per block: the march reads them at every face
  __shared__ __align__(16) KParams sP;
  const int tid = threadIdx.x;
  const int tx = tid % SX, ty = tid / SX;
  const int lx = tx - 1, ly = DIM >= 2 ? ty - 1 : 0;
  const bool row_t = ty >= 1 && ty <= BS;
  const bool col_t = tx >= 1 && tx <= BS;
  const bool tile_t = row_t && col_t;
  auto ring = [&](int plane) -> float* { return sW + ((plane + 6) % 3) * 6 * SWN; };

  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int slot = __ldg(list + i);
    const int g = bt_at(bt, slot, GRID_WORD);
    const double dt = clks[g].dt;
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
    const bool g_coarse = gface >= 0 && gnb == -1;
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
    }
    const int fine0 = bt_at(bt, slot, FINE_WORD);
    if (fine0 < 0 || fbuf == nullptr) fine = 0;
    auto matched = [&](int f, int cidx, float* F) {
      const float4* q = fbuf + ((size_t)(fine0 + __popc(fine & ((1u << f) - 1u))) * FC + cidx) * 2;
      const float4 a = __ldg(q), b = __ldg(q + 1);
      F[0] = a.x; F[1] = a.y; F[2] = a.z; F[3] = a.w;
      F[4] = b.x; F[5] = b.y; F[6] = b.z; F[7] = b.w;
    };
    const int zlo_nb = DIM == 3 ? bt_at(bt, slot, 10) : 0, zhi_nb = DIM == 3 ? bt_at(bt, slot, 11) : 0;

    float zhi_prev[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float ph_prev = 0.f;

    auto load_plane = [&](int pl) {
      float* dst = ring(pl);
      const size_t zb = (size_t)slot * BG<DIM>::WN + (DIM == 3 ? (size_t)(pl + NG) * SWN : 0);
      for (int t = tid; t < SWN; t += SNT) {
        const float4 a = __ldg(w1 + zb + t), b = __ldg(w2 + zb + t);
        dst[0 * SWN + t] = a.x;
        dst[1 * SWN + t] = a.y;
        dst[2 * SWN + t] = a.z;
        dst[3 * SWN + t] = a.w;
        dst[4 * SWN + t] = b.x;
        dst[5 * SWN + t] = b.y;
      }
    };
    if constexpr (DIM == 3) {
      load_plane(-2);
      load_plane(-1);
    }
    // 3D: planes -1 .. 16, the first and last the z ghosts; 2D: the one plane.
    const int jb = DIM == 3 ? -1 : 0, je = DIM == 3 ? BS : 0;
    for (int j = jb; j <= je; j++) {
      load_plane(DIM == 3 ? j + 1 : 0);
      __syncthreads();
      const float* pj = ring(DIM == 3 ? j : 0);
      const bool zghost = DIM == 3 && (j == -1 || j == BS);
      const int znb = j == -1 ? zlo_nb : zhi_nb;  // (meaningful on the z ghost planes)

      // the predictor at plane j
      float c[7];
      read_w6(pj, lx, ly, c);
      with_cs(c, P);
      float su[DIM][6], sd[DIM][6];
      float conv = 0.f, jump = 0.f;
      {
        float m[7], p[7];
        read_w6(pj, lx - 1, ly, m);
        read_w6(pj, lx + 1, ly, p);
        axis_edges<R, ISEN>(m, m, c, p, p, P.inv_gamma, su[0], sd[0]);
        conv += p[1] - m[1];
        jump = fmaxf(jump, fabsf(p[4] - m[4]) / fminf(p[4], m[4]));
        if constexpr (DIM >= 2) {
          read_w6(pj, lx, ly - 1, m);
          read_w6(pj, lx, ly + 1, p);
          axis_edges<R, ISEN>(m, m, c, p, p, P.inv_gamma, su[1], sd[1]);
          conv += p[2] - m[2];
          jump = fmaxf(jump, fabsf(p[4] - m[4]) / fminf(p[4], m[4]));
        }
        if constexpr (DIM == 3) {
          read_w6(ring(j - 1), lx, ly, m);
          read_w6(ring(j + 1), lx, ly, p);
          axis_edges<R, ISEN>(m, m, c, p, p, P.inv_gamma, su[2], sd[2]);
          conv += p[3] - m[3];
          jump = fmaxf(jump, fabsf(p[4] - m[4]) / fminf(p[4], m[4]));
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
        if (zghost && znb == -1) {
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
          face_state(gq, inc, 1.f, zhi_prev);
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
      __syncthreads();

      const int lz = DIM == 3 ? j : 0;
      if (tile_plane) {
        if (row_t && tx >= 1) {
          // the x face below cell lx (lx = 0 .. 16)
          float L[7], Rr[7], F[8];
#pragma unroll
          for (int v = 0; v < 7; v++) L[v] = sFace[v * SPN + tid - 1];
          face_state(pr, sd[0], -1.f, Rr);
          riemann<0>(L, Rr, P, F);
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
            riemann<1>(L, Rr, P, F);
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
          riemann<2>(zhi_prev, Rr, P, Fz);
          if ((j == 0 && (fine & 16u)) || (j == BS && (fine & 32u))) matched(j == 0 ? 4 : 5, lx + BS * ly, Fz);
        }
      }
      __syncthreads();

      if (tile_t) {
        if constexpr (DIM == 3) {
          if (j >= 1) {
            // plane j - 1 is complete: its upper z face is Fz
#pragma unroll
            for (int v = 0; v < 8; v++) acc[v] -= Fz[v];
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
            if constexpr (DIM == 3) a += Fz[v];
            acc[v] = a;
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
        if (!(j == -1 && zlo_nb <= -2)) face_state(pr, su[2], 1.f, zhi_prev);
      }
    }
  }
}

}  // namespace amrk

// ---------------------------------------------------------------------------------------------
// Host launchers.

namespace {
int grid_for(int n, int per_sm) {
  int g = 148 * per_sm;
  if (n < g) g = n;
  return g < 1 ? 1 : g;
}
}  // namespace

#define SHZ_RECON_SWITCH(recon, ISEN, CALL)                                  \
  switch (recon) {                                                           \
    case R_MINMOD: { constexpr int R = R_MINMOD; CALL; break; }             \
    case R_MC: { constexpr int R = R_MC; CALL; break; }                     \
    case R_VANLEER: { constexpr int R = R_VANLEER; CALL; break; }           \
    default: { constexpr int R = R_KOREN; CALL; break; }                    \
  }

cudaError_t amr_launch_assemble(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                                unsigned* rates, int rslot, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int g = grid_for(n, 4);
  if (L.ndim == 3) {
    SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_assemble<3, R><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, rates, rslot)))
  } else {
    SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_assemble<2, R><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, rates, rslot)))
  }
  return cudaGetLastError();
}

cudaError_t amr_launch_predict(const AmrLaunch& L, const int* list, int n, const DevClock* clks, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int g = grid_for(n, 4);
  if (L.ndim == 3) {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_predict<3, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, L.w1, L.w2, L.p1, L.p2, clks))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_predict<3, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, L.w1, L.w2, L.p1, L.p2, clks))) }
  } else {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_predict<2, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, L.w1, L.w2, L.p1, L.p2, clks))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_predict<2, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, L.w1, L.w2, L.p1, L.p2, clks))) }
  }
  return cudaGetLastError();
}

cudaError_t amr_launch_update(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, float4* o1,
                              float4* o2, const DevClock* clks, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int g = grid_for(n, 4);
  if (L.ndim == 3) {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_update<3, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, L.p1, L.p2, o1, o2, clks))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_update<3, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, L.p1, L.p2, o1, o2, clks))) }
  } else {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_update<2, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, L.p1, L.p2, o1, o2, clks))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_update<2, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, L.p1, L.p2, o1, o2, clks))) }
  }
  return cudaGetLastError();
}

namespace {
template <int DIM, int R, bool ISEN>
cudaError_t sweep_one(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, float4* o1,
                      float4* o2, const DevClock* clks, cudaStream_t s) {
  auto k = amrk::amr_sweep<DIM, R, ISEN>;
  // (set once per instantiation; an attribute call is not a stream operation, so a first call
  // inside a stream capture is fine)
  static const cudaError_t attr = [&] {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)amrk::SWEEP_SMEM);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    return e;
  }();
  if (attr != cudaSuccess) return attr;
  k<<<grid_for(n, 2), amrk::SNT, amrk::SWEEP_SMEM, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, o1, o2, clks, L.fbuf);
  return cudaGetLastError();
}
}  // namespace

cudaError_t amr_launch_fine_flux(const AmrLaunch& L, const int* flist, int nf, const DevClock* clks, cudaStream_t s) {
  if (nf <= 0) return cudaSuccess;
  const long long cells = (long long)nf * (L.ndim == 3 ? 256 : 16);
  const int g = (int)std::min<long long>((cells + amrk::NT - 1) / amrk::NT, 148LL * 8);
  if (L.ndim == 3) {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_fine_flux<3, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, flist, nf, L.w1, L.w2, clks, L.fbuf))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_fine_flux<3, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, flist, nf, L.w1, L.w2, clks, L.fbuf))) }
  } else {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, (amrk::amr_fine_flux<2, R, true><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, flist, nf, L.w1, L.w2, clks, L.fbuf))) }
    else { SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_fine_flux<2, R, false><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, flist, nf, L.w1, L.w2, clks, L.fbuf))) }
  }
  return cudaGetLastError();
}

cudaError_t amr_launch_sweep(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, float4* o1,
                             float4* o2, const DevClock* clks, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if (L.ndim == 3) {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, return (sweep_one<3, R, true>(L, list, n, u1, u2, o1, o2, clks, s))) }
    else { SHZ_RECON_SWITCH(L.recon, false, return (sweep_one<3, R, false>(L, list, n, u1, u2, o1, o2, clks, s))) }
  } else {
    if (L.isen) { SHZ_RECON_SWITCH(L.recon, true, return (sweep_one<2, R, true>(L, list, n, u1, u2, o1, o2, clks, s))) }
    else { SHZ_RECON_SWITCH(L.recon, false, return (sweep_one<2, R, false>(L, list, n, u1, u2, o1, o2, clks, s))) }
  }
  return cudaSuccess;
}

cudaError_t amr_launch_flag(const AmrLaunch& L, const int* list, int n, float* flags, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int g = grid_for(n, 4);
  if (L.ndim == 3) amrk::amr_flag<3><<<g, amrk::NT, 0, s>>>(list, n, L.w1, L.w2, flags);
  else amrk::amr_flag<2><<<g, amrk::NT, 0, s>>>(list, n, L.w1, L.w2, flags);
  return cudaGetLastError();
}

cudaError_t amr_launch_regrid(const AmrLaunch& L, const int* rg, const int* list, int n, const float4* u1, const float4* u2,
                              float4* o1, float4* o2, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int g = grid_for(n, 4);
  if (L.ndim == 3) {
    SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_regrid<3, R><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, rg, list, n, u1, u2, L.w1, L.w2, o1, o2)))
  } else {
    SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_regrid<2, R><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, rg, list, n, u1, u2, L.w1, L.w2, o1, o2)))
  }
  return cudaGetLastError();
}

// The clocks of many grids at once, one thread each: as clock_kernel (sweep.cu), reading grid
// g's rate from rates[2 g + rslot] and clearing the other slot for the next step; a grid that
// has taken max_steps steps holds.
__global__ void clock_multi_kernel(DevClock* __restrict__ clks, unsigned* __restrict__ rates, int rslot, int ngrids) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngrids) return;
  DevClock& c = clks[g];
  const float rate = __uint_as_float(rates[2 * g + rslot]);
  rates[2 * g + (rslot ^ 1)] = 0u;
  const double t = c.t;
  double dt = c.cfl_dx / fmax((double)rate, 1e-30);
  if (!(rate == rate) || isinf(rate)) c.bad = 1;
  dt = fmin(dt, c.dt_max);
  const double te = c.t_end;
  if (te < HUGE_VAL) {
    const double rem = te - t;
    if (rem <= 1e-12 * fabs(te)) dt = 0.0;
    else dt = fmin(dt, rem);
  }
  if (c.bad || c.steps >= c.max_steps) dt = 0.0;
  c.dt = dt;
  c.held = dt > 0.0 ? 0 : 1;
  if (dt > 0.0) {
    c.t = t + dt;
    c.steps += 1;
    c.last_dt = dt;
  }
}

cudaError_t launch_clock_multi(DevClock* clks, unsigned* rates, int rslot, int ngrids, cudaStream_t s) {
  if (ngrids <= 0) return cudaSuccess;
  clock_multi_kernel<<<(ngrids + 127) / 128, 128, 0, s>>>(clks, rates, rslot, ngrids);
  return cudaGetLastError();
}

int amr_diag_blocks(int n) { return grid_for(n, 2); }

cudaError_t amr_launch_diag(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, double* part,
                            double* out, cudaStream_t s) {
  const int g = amr_diag_blocks(n);
  if (L.ndim == 3) amrk::amr_diag<3><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, part);
  else amrk::amr_diag<2><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, part);
  amrk::amr_diag_final<<<1, 32, 0, s>>>(part, g, out);
  return cudaGetLastError();
}

cudaError_t amr_launch_ghost_map(const AmrLaunch& L, int slot, int* out, cudaStream_t s) {
  if (L.ndim == 3) amrk::amr_ghost_map<3><<<32, 256, 0, s>>>(L.bt, slot, out);
  else amrk::amr_ghost_map<2><<<2, 256, 0, s>>>(L.bt, slot, out);
  return cudaGetLastError();
}

}  // namespace shz
