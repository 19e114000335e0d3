// The passes of one step on the adaptive block grid, as persistent work-list kernels, and those
// of the refinement check. One step is three or four kernels, captured in a CUDA graph by the
// host:
//   1. amr_assemble over the leaves (with two_pass, every block): primitives with ghost fill, and
//      the leaves' rate / dx maximum.
//   2. clock_multi_kernel: dt.
//   3. amr_fine_flux (amr_sweep.cu) over the faces whose same-level neighbour is refined: the
//      mean fine fluxes (only when the mesh has such faces).
//   4. amr_sweep (amr_sweep.cu) over the leaves: half steps, fluxes and the update, in one pass
//      over the primitives, the matched faces' fluxes read from the buffer step 3 filled.
// The reference's own pass structure is kept beside it as a cross-check (two_pass,
// amr_twopass.cu): amr_predict writes the half steps to their atlas and amr_update reads them.
// This follows the reference's AmrSim.encodeSteps (src/amr/amr_sim.ts:2709-2946). Every kernel
// walks a device list of block slots with a fixed grid of CTAs, one block at a time per CTA.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>

#include "amr_device.cuh"
#include "diag_ext.cuh"

namespace shz {
namespace amrk {

// The coarse-cell table of the assemble: for each face of a block whose neighbour is one level
// coarser, the state and prolongation slopes of the coarse cells its ghosts lie over (8 x 8 in
// 3D, 8 in 2D; the two ghost layers are one coarse layer), 33 floats each: uc, three slopes, the
// common scale-back factor. Every fine ghost over a coarse cell reads the same entry.
constexpr int TAB_VALS = 33;
template <int DIM>
struct Tab {
  static constexpr int CPF = DIM == 3 ? 64 : 8;  // coarse cells per face
  static constexpr size_t BYTES = (size_t)2 * DIM * CPF * TAB_VALS * sizeof(float);
};
// The second pass's table of the edge and corner ghosts that reach a coarser leaf through a
// same-level neighbour: 8 coarse cells along each of the 12 edges (a coarse cell spans 2 fine
// texels along the edge and both ghost layers across it) and one per corner in 3D; one per corner
// in 2D. Entries in the same layout as the face table's.
template <int DIM>
struct EdgeTab {
  static constexpr int N = DIM == 3 ? 12 * (BS / 2) + 8 : 4;
  static constexpr size_t BYTES = (size_t)N * TAB_VALS * sizeof(float);
};

__device__ __forceinline__ void tab_store(float* e, const Cons& uc, const Slopes& sl) {
  const float4 v[8] = {uc.a, uc.b, sl.s[0].a, sl.s[0].b, sl.s[1].a, sl.s[1].b, sl.s[2].a, sl.s[2].b};
#pragma unroll
  for (int k = 0; k < 8; k++) {
    e[4 * k] = v[k].x;
    e[4 * k + 1] = v[k].y;
    e[4 * k + 2] = v[k].z;
    e[4 * k + 3] = v[k].w;
  }
  e[32] = sl.f;
}
__device__ __forceinline__ void tab_load(const float* e, Cons& uc, Slopes& sl) {
  float4 v[8];
#pragma unroll
  for (int k = 0; k < 8; k++) v[k] = make_float4(e[4 * k], e[4 * k + 1], e[4 * k + 2], e[4 * k + 3]);
  uc = Cons{v[0], v[1]};
  sl.s[0] = Cons{v[2], v[3]};
  sl.s[1] = Cons{v[4], v[5]};
  sl.s[2] = Cons{v[6], v[7]};
  sl.f = e[32];
}

// The texels of a block's primitive region outside its own cells (the two ghost layers), numbered
// 0 .. WN - CB - 1: in 3D the four ghost planes z = -2, -1, 16, 17 whole, then the ring of each
// plane z = 0 .. 15; in 2D the ring of the one plane. A ring (20^2 - 16^2 = 144 texels) is the rows
// y = -2, -1, then y = 16, 17, then x = -2, -1, 16, 17 of the rows y = 0 .. 15.
__device__ __forceinline__ void ring_texel(int k, int& x, int& y) {
  if (k < 2 * PAD) {
    y = k / PAD - NG;
    x = k % PAD - NG;
  } else if (k < 4 * PAD) {
    k -= 2 * PAD;
    y = k / PAD + BS;
    x = k % PAD - NG;
  } else {
    k -= 4 * PAD;
    y = k >> 2;
    const int c = k & 3;
    x = c < 2 ? c - NG : c - 2 + BS;
  }
}
template <int DIM>
__device__ __forceinline__ void shell_texel(int i, int* l) {
  constexpr int RING = PAD * PAD - BS * BS;
  if (DIM == 2) {
    ring_texel(i, l[0], l[1]);
    l[2] = 0;
  } else if (i < 2 * NG * PAD * PAD) {
    const int p = i / (PAD * PAD), r = i % (PAD * PAD);
    l[2] = p < NG ? p - NG : p - NG + BS;
    l[0] = r % PAD - NG;
    l[1] = r / PAD - NG;
  } else {
    const int j = i - 2 * NG * PAD * PAD;
    l[2] = j / RING;
    ring_texel(j % RING, l[0], l[1]);
  }
}

// The neighbour direction of texel l: codes 0, 1, 2 per axis for below, inside and above the
// block, d = x + 3 y + 9 z.
template <int DIM>
__device__ __forceinline__ int dir_code(const int* l) {
  return (l[0] < 0 ? 0 : l[0] >= BS ? 2 : 1) + 3 * (l[1] < 0 ? 0 : l[1] >= BS ? 2 : 1) +
         (DIM == 3 ? 9 * (l[2] < 0 ? 0 : l[2] >= BS ? 2 : 1) : 0);
}

// Edge-table entries of neighbour direction d (codes 0, 1, 2 per axis for below, inside and above
// the block, d = x + 3 y + 9 z) when its ghosts reach a coarser leaf through another block: a 3D
// edge (one axis inside) spans 8 coarse cells, a corner one.
template <int DIM>
__device__ __forceinline__ int edge_entries(int d) {
  const int inside = (d % 3 == 1) + ((d / 3) % 3 == 1) + (DIM == 3 ? (d / 9 == 1) : 0);
  return (DIM == 3 && inside == 1) ? BS / 2 : 1;
}

// A ghost whose source is a cell of a same-level leaf (not a parent, whose cells are restricted,
// and not a leaf part way through a longer step, whose half step is read): one load gives it.
template <bool BINS>
__device__ __forceinline__ bool plain_src(const int* __restrict__ bt, const int* __restrict__ bins, const Src& s) {
  return s.kind == 0 && leaf_of(bt, s.slot) && !(BINS && mid_block(bt, bins, s.slot));
}

// 1. Primitives of every block in the list with two ghost layers; the rate / dx maximum over the
// leaves' own cells (assemble.wgsl:78-154; PER_DX in clock.wgsl). MINB: the CTAs per SM the
// register budget is planned for (the autotuner's variant): more CTAs hide the gather's latency,
// fewer registers spill on the prolongation path of coarse ghosts. Ghosts beyond a coarser
// block's face take their coarse cell's state and slopes from the block's table (built first,
// once per coarse cell); with per_texel (the two-pass mode, the reference's structure) each
// ghost forms them itself. Both give the same numbers.
// With per-block timesteps (BINS, the bin table `bins`), a source leaf part way through its step
// gives its half-step state from p1, p2 (amr/assemble.wgsl with <mid>, amr/mid_on.wgsl), and each
// leaf's own rate / dx also goes to brate[slot] for its bin.
// REST: the second pass of the split form, after amr_assemble_plain: only the ghosts whose source
// is not a same-level leaf's cell (restriction, prolongation, half steps); no rate.
template <int DIM, int R, int MINB, bool BINS, bool REST>
__global__ void __launch_bounds__(NT, MINB) amr_assemble(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                   const int* __restrict__ list, int n, const float4* __restrict__ u1,
                                                   const float4* __restrict__ u2, float4* __restrict__ w1,
                                                   float4* __restrict__ w2, unsigned* __restrict__ rates, int rslot,
                                                   int per_texel, const float4* __restrict__ p1,
                                                   const float4* __restrict__ p2, const int* __restrict__ bins,
                                                   float* __restrict__ brate) {
  using T = Tab<DIM>;
  __shared__ float sRed[NT / 32];
  __shared__ unsigned sPlain;  // REST: bit d set when the ghosts of neighbour direction d are plain
  __shared__ int sEdge[27];    // REST: first edge-table entry of direction d, or -1
  __shared__ int sEdgeN;       // REST: edge-table entries of this block
  extern __shared__ __align__(16) float sTab[];
  float* const sEdgeTab = sTab + (size_t)2 * DIM * T::CPF * TAB_VALS;  // REST and !per_texel only
  constexpr bool EDGES = REST;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    float rmax = 0.f;
    const int slot = __ldg(list + i);
    const int g = bt_at(bt, slot, GRID_WORD);
    const KParams& P = gp[g];
    const int nr = P.n[0];
    const bool leaf = leaf_of(bt, slot);
    const float inv_dx = (float)(ldexp(1.0, bt_at(bt, slot, 0)) / P.dx);
    unsigned cmask = 0;
    if (!per_texel)
#pragma unroll
      for (int f = 0; f < 2 * DIM; f++)
        if (bt_at(bt, slot, 6 + f) == -1) cmask |= 1u << f;
    if (REST && threadIdx.x < 32) {
      // Which neighbour directions' ghosts the first pass filled: every texel of a direction
      // resolves through the same hops to the same kind of source (the hops move an out-of-range
      // axis into the block whatever its ghost layer), so one texel per direction decides.
      const int d = threadIdx.x;
      bool plain = false;
      int cnt = 0;  // edge-table entries of direction d
      if (d < (DIM == 3 ? 27 : 9) && d != (DIM == 3 ? 13 : 4)) {
        const int l[3] = {d % 3 == 0 ? -1 : d % 3 == 2 ? BS : 0, (d / 3) % 3 == 0 ? -1 : (d / 3) % 3 == 2 ? BS : 0,
                          DIM == 3 ? (d / 9 == 0 ? -1 : d / 9 == 2 ? BS : 0) : 0};
        const Src sd = ghost_src_any<DIM>(bt, slot, l);
        plain = plain_src<BINS>(bt, bins, sd);
        // a coarser leaf reached through another block (an edge or corner direction): its coarse
        // cells go into the edge table, 8 along a 3D edge, one at a corner
        if (EDGES && !per_texel && sd.kind == 1 && sd.from != slot) cnt = edge_entries<DIM>(d);
      }
      const unsigned m = __ballot_sync(0xffffffffu, plain);
      if (d == 0) sPlain = m;
      if (EDGES) {
        int base = cnt;  // inclusive scan of the counts over the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, base, o);
          if (d >= o) base += v;
        }
        if (d < 27) sEdge[d] = cnt ? base - cnt : -1;
        if (d == 31) sEdgeN = base;
      }
    }
    if (EDGES) __syncthreads();  // the edge directions, before their table is built
    const int nedge = EDGES ? sEdgeN : 0;
    if (cmask || nedge) {
      // the table of this block's coarse faces (the previous block's reads of it ended at the
      // barriers of its rate maximum), then the edge table's entries
      const int nface = __popc(cmask) * T::CPF;
      for (int idx = threadIdx.x; idx < nface + nedge; idx += NT) {
        int from = slot, m[3] = {0, 0, 0}, cs;
        float* dst;
        if (idx < nface) {
          const int k = idx / T::CPF, c = idx % T::CPF;
          unsigned mk = cmask;
          for (int q = 0; q < k; q++) mk &= mk - 1;
          const int f = __ffs(mk) - 1;
          const int a = f >> 1;
          m[a] = (f & 1) ? BS : -1;
          if (DIM == 3) {
            m[(a + 1) % 3] = 2 * (c % 8);
            m[(a + 2) % 3] = 2 * (c / 8);
          } else {
            m[1 - a] = 2 * c;
          }
          cs = bt_at(bt, slot, 20 + f);
          dst = sTab + (size_t)(f * T::CPF + c) * TAB_VALS;
        } else {
          const int e = idx - nface;
          int d = 0;
          while (d < 26 && !(sEdge[d] >= 0 && e >= sEdge[d] && e < sEdge[d] + edge_entries<DIM>(d))) d++;
          // the direction's representative texel, at the entry's coarse cell along a 3D edge
          int l[3] = {d % 3 == 0 ? -1 : d % 3 == 2 ? BS : 0, (d / 3) % 3 == 0 ? -1 : (d / 3) % 3 == 2 ? BS : 0,
                      DIM == 3 ? (d / 9 == 0 ? -1 : d / 9 == 2 ? BS : 0) : 0};
          if (DIM == 3) {
            const int c = d % 3 == 1 ? 0 : (d / 3) % 3 == 1 ? 1 : d / 9 == 1 ? 2 : -1;
            if (c >= 0) l[c] = 2 * (e - sEdge[d]);
          }
          const Src se = ghost_src_any<DIM>(bt, slot, l);
          from = se.from;
          m[0] = se.l[0];
          m[1] = se.l[1];
          m[2] = se.l[2];
          cs = se.slot;
          dst = sEdgeTab + (size_t)e * TAB_VALS;
        }
        Cons uc;
        Slopes sl;
        int par[3];
        if (BINS && mid_block(bt, bins, cs)) coarse_cell_mid<DIM, R>(P, bt, p1, p2, nr, from, m, cs, uc, sl, par);
        else coarse_cell<DIM, R>(bt, u1, u2, nr, from, m, cs, P.rho_floor, uc, sl, par);
        tab_store(dst, uc, sl);
      }
    }
    if (cmask || REST) __syncthreads();  // (REST: also the edge table)
    // the block's own cells (a parent's restricted from its children), with the rate maximum
#pragma unroll 4
    for (int t = threadIdx.x; t < (REST ? 0 : BG<DIM>::CB); t += NT) {
      const int l[3] = {t & (BS - 1), (t >> 4) & (BS - 1), DIM == 3 ? t >> 8 : 0};
      const Cons u = u_at<DIM>(bt, u1, u2, slot, l);
      float w[7];
      prim_from_cons(u.a, u.b, P, 1.f, 1.f, 1.f, w);
      const size_t o = (size_t)slot * BG<DIM>::WN + wtex<DIM>(l);
      w1[o] = make_float4(w[0], w[1], w[2], w[3]);
      w2[o] = make_float4(w[4], w[5], w[6], 0.f);
      if (leaf) rmax = fmaxf(rmax, rate_guard_f(fabsf(w[1]) + fabsf(w[2]) + fabsf(w[3]) + P.signal * w[6]) * inv_dx);
    }
    // the ghost layers, each from its source
    for (int i = threadIdx.x; i < BG<DIM>::WN - BG<DIM>::CB; i += NT) {
      int l[3];
      shell_texel<DIM>(i, l);
      if (REST && ((sPlain >> dir_code<DIM>(l)) & 1u)) continue;
      const Src s = ghost_src_any<DIM>(bt, slot, l);
      Cons u;
      if (s.kind == 0) {
        if (BINS && mid_block(bt, bins, s.slot)) u = mid_cons<DIM>(P, p1, p2, s.slot, s.l);
        else u = u_at<DIM>(bt, u1, u2, s.slot, s.l);
      } else if ((cmask && s.from == slot) || (EDGES && nedge && sEdge[dir_code<DIM>(l)] >= 0)) {
        // a ghost beyond a coarser leaf whose coarse cell is in a table: this block's own coarse
        // face's, or (an edge or corner ghost reached through another block) the edge table's
        const float* ent;
        if (cmask && s.from == slot) {
          int a = 0;
#pragma unroll
          for (int q = 0; q < DIM; q++)
            if (s.l[q] < 0 || s.l[q] >= BS) a = q;
          const int f = 2 * a + (s.l[a] >= BS ? 1 : 0);
          const int c = DIM == 3 ? (s.l[(a + 1) % 3] >> 1) + 8 * (s.l[(a + 2) % 3] >> 1) : (s.l[1 - a] >> 1);
          ent = sTab + (size_t)(f * T::CPF + c) * TAB_VALS;
        } else {
          // along a 3D edge, the coarse cell under the texel's position on the axis inside
          const int d = dir_code<DIM>(l);
          const int in = DIM == 3 ? (d % 3 == 1 ? l[0] : (d / 3) % 3 == 1 ? l[1] : d / 9 == 1 ? l[2] : 0) : 0;
          ent = sEdgeTab + (size_t)(sEdge[d] + (in >> 1)) * TAB_VALS;
        }
        Cons uc;
        Slopes sl;
        tab_load(ent, uc, sl);
        const int par[3] = {s.l[0] & 1, s.l[1] & 1, DIM == 3 ? (s.l[2] & 1) : 0};
        u = prolong_child(uc, sl, par);
      } else if (BINS && mid_block(bt, bins, s.slot)) {
        u = from_coarse_mid<DIM, R>(P, bt, p1, p2, nr, s.from, s.l, s.slot);
      } else {
        u = from_coarse<DIM, R>(bt, u1, u2, nr, s.from, s.l, s.slot, P.rho_floor);
      }
      u.a.y *= s.flip[0];
      u.a.z *= s.flip[1];
      u.a.w *= s.flip[2];
      float w[7];
      prim_from_cons(u.a, u.b, P, 1.f, 1.f, 1.f, w);
      const size_t o = (size_t)slot * BG<DIM>::WN + wtex<DIM>(l);
      w1[o] = make_float4(w[0], w[1], w[2], w[3]);
      w2[o] = make_float4(w[4], w[5], w[6], 0.f);
    }
    if (REST) {
      __syncthreads();  // the coarse table is rebuilt for the next block
      continue;
    }
    const float m = block_max(rmax, sRed);
    if (threadIdx.x == 0 && leaf) {
      atomicMax(rates + 2 * g + rslot, __float_as_uint(m));
      if (BINS && brate) brate[slot] = m;
    }
  }
}

// 1a. The first pass of the split assemble: what needs no more than one load of a cell per texel,
// at the occupancy of a light kernel (4 CTAs per SM): every block's own cells, with the rate
// maximum, and the ghosts whose source is a same-level leaf's cell (its face, edge and corner
// neighbours at its own level, and its images across the domain's faces). The rest of the ghosts
// are the second pass's (amr_assemble with REST). Every texel gets the same numbers as in the
// one-pass kernel: the same load, velocity signs and prim_from_cons.
template <int DIM, bool BINS>
__global__ void __launch_bounds__(NT, 4) amr_assemble_plain(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                        const int* __restrict__ list, int n, const float4* __restrict__ u1,
                                                        const float4* __restrict__ u2, float4* __restrict__ w1,
                                                        float4* __restrict__ w2, unsigned* __restrict__ rates, int rslot,
                                                        const int* __restrict__ bins, float* __restrict__ brate) {
  __shared__ float sRed[NT / 32];
  constexpr int NS = BG<DIM>::WN - BG<DIM>::CB;
  constexpr int U = 1;  // shell texels a thread resolves, then loads together (more spill in 3D)
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    float rmax = 0.f;
    const int slot = __ldg(list + i);
    const int g = bt_at(bt, slot, GRID_WORD);
    const KParams& P = gp[g];
    const bool leaf = leaf_of(bt, slot);
    const float inv_dx = (float)(ldexp(1.0, bt_at(bt, slot, 0)) / P.dx);
    if (leaf) {
      // a leaf's own cells: u_at's load of its own cell
#pragma unroll 4
      for (int t = threadIdx.x; t < BG<DIM>::CB; t += NT) {
        const int l[3] = {t & (BS - 1), (t >> 4) & (BS - 1), DIM == 3 ? t >> 8 : 0};
        const size_t c = (size_t)slot * BG<DIM>::CB + t;
        const float4 ua = __ldg(u1 + c), ub = __ldg(u2 + c);
        float w[7];
        prim_from_cons(ua, ub, P, 1.f, 1.f, 1.f, w);
        const size_t o = (size_t)slot * BG<DIM>::WN + wtex<DIM>(l);
        w1[o] = make_float4(w[0], w[1], w[2], w[3]);
        w2[o] = make_float4(w[4], w[5], w[6], 0.f);
        rmax = fmaxf(rmax, rate_guard_f(fabsf(w[1]) + fabsf(w[2]) + fabsf(w[3]) + P.signal * w[6]) * inv_dx);
      }
    } else {
      // a parent's (the two-pass form assembles every block): restricted from its children
      for (int t = threadIdx.x; t < BG<DIM>::CB; t += NT) {
        const int l[3] = {t & (BS - 1), (t >> 4) & (BS - 1), DIM == 3 ? t >> 8 : 0};
        const Cons u = u_at<DIM>(bt, u1, u2, slot, l);
        float w[7];
        prim_from_cons(u.a, u.b, P, 1.f, 1.f, 1.f, w);
        const size_t o = (size_t)slot * BG<DIM>::WN + wtex<DIM>(l);
        w1[o] = make_float4(w[0], w[1], w[2], w[3]);
        w2[o] = make_float4(w[4], w[5], w[6], 0.f);
      }
    }
    for (int i0 = threadIdx.x; i0 < NS; i0 += U * NT) {
      long long src[U];
      int dst[U];  // the texel (13 bits), and bits 13-15: the velocity components whose sign flips
#pragma unroll
      for (int q = 0; q < U; q++) {
        const int k = i0 + q * NT;
        src[q] = -1;
        dst[q] = 0;
        if (k < NS) {
          int l[3];
          shell_texel<DIM>(k, l);
          const Src s = ghost_src_any<DIM>(bt, slot, l);
          if (plain_src<BINS>(bt, bins, s)) {
            // u_at's index for a leaf, clamped as there
            const int c[3] = {min(max(s.l[0], 0), BS - 1), min(max(s.l[1], 0), BS - 1),
                              DIM == 3 ? min(max(s.l[2], 0), BS - 1) : 0};
            src[q] = (long long)s.slot * BG<DIM>::CB + cell_ix<DIM>(c);
            dst[q] = wtex<DIM>(l) | (s.flip[0] < 0.f ? 1 << 13 : 0) | (s.flip[1] < 0.f ? 1 << 14 : 0) |
                     (s.flip[2] < 0.f ? 1 << 15 : 0);
          }
        }
      }
      float4 a[U], b[U];
#pragma unroll
      for (int q = 0; q < U; q++) {
        if (src[q] >= 0) {
          a[q] = __ldg(u1 + src[q]);
          b[q] = __ldg(u2 + src[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < U; q++) {
        if (src[q] < 0) continue;
        Cons u{a[q], b[q]};
        u.a.y *= (dst[q] >> 13) & 1 ? -1.f : 1.f;
        u.a.z *= (dst[q] >> 14) & 1 ? -1.f : 1.f;
        u.a.w *= (dst[q] >> 15) & 1 ? -1.f : 1.f;
        float w[7];
        prim_from_cons(u.a, u.b, P, 1.f, 1.f, 1.f, w);
        const size_t o = (size_t)slot * BG<DIM>::WN + (dst[q] & 0x1FFF);
        w1[o] = make_float4(w[0], w[1], w[2], w[3]);
        w2[o] = make_float4(w[4], w[5], w[6], 0.f);
      }
    }
    const float m = block_max(rmax, sRed);
    if (threadIdx.x == 0 && leaf) {
      atomicMax(rates + 2 * g + rslot, __float_as_uint(m));
      if (BINS && brate) brate[slot] = m;
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

// The extended channels (diag_ext.cuh) over the leaves: cell centres from the box centre, each
// block's cells of its own level's size (amr/grid.wgsl:172-177 blk_pos); a 2D grid in z = 0.
template <int DIM>
__global__ void __launch_bounds__(NT) amr_diag_ext(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                   const int* __restrict__ list, int n, const float4* __restrict__ u1,
                                                   const float4* __restrict__ u2, double* __restrict__ part) {
  dext::Ext e;
  e.init();
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int slot = __ldg(list + i);
    const KParams& P = gp[bt_at(bt, slot, GRID_WORD)];
    const double dx = P.dx / ldexp(1.0, bt_at(bt, slot, 0));
    const double dv = DIM == 3 ? dx * dx * dx : dx * dx;
    const double half = 0.5 * P.n[0] * BS * P.dx;  // half the box: n[0] root blocks of BS cells
    const int c0 = bt_at(bt, slot, 1), c1 = bt_at(bt, slot, 2), c2 = bt_at(bt, slot, 3);
    for (int t = threadIdx.x; t < BG<DIM>::CB; t += NT) {
      const int l0 = t % BS, l1 = (t / BS) % BS, l2 = DIM == 3 ? t / (BS * BS) : 0;
      const double x = (c0 * BS + l0 + 0.5) * dx - half;
      const double y = (c1 * BS + l1 + 0.5) * dx - half;
      const double z = DIM == 3 ? (c2 * BS + l2 + 0.5) * dx - half : 0.0;
      const size_t o = (size_t)slot * BG<DIM>::CB + t;
      e.cell(__ldg(u1 + o), __ldg(u2 + o), P, dv, x, y, z);
    }
  }
  dext::block_reduce(e, part + (size_t)blockIdx.x * dext::N);
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

}  // namespace amrk

// ---------------------------------------------------------------------------------------------
// Host launchers.

namespace {
template <int DIM, int R, int MINB, bool BINS = false, bool REST = false>
cudaError_t assemble_t(const AmrLaunch& L, int g, const int* list, int n, const float4* u1, const float4* u2,
                       unsigned* rates, int rslot, cudaStream_t s, const int* bins = nullptr, float* brate = nullptr) {
  auto k = amrk::amr_assemble<DIM, R, MINB, BINS, REST>;
  // the coarse-face table, and in the second pass of the split form also the edge table
  constexpr size_t TB = amrk::Tab<DIM>::BYTES + (REST ? amrk::EdgeTab<DIM>::BYTES : 0);
  // (set once per instantiation; not a stream operation)
  static const cudaError_t attr = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TB);
  if (attr != cudaSuccess) return attr;
  const size_t smem = L.per_texel ? 0 : TB;
  k<<<g, amrk::NT, smem, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, rates, rslot, L.per_texel ? 1 : 0, L.p1, L.p2,
                              bins, brate);
  return cudaGetLastError();
}
template <int MINB>
cudaError_t assemble_v(const AmrLaunch& L, int g, const int* list, int n, const float4* u1, const float4* u2,
                       unsigned* rates, int rslot, cudaStream_t s) {
  if (L.ndim == 3) {
    SHZ_RECON_SWITCH(L.recon, false, return (assemble_t<3, R, MINB>(L, g, list, n, u1, u2, rates, rslot, s)))
  } else {
    SHZ_RECON_SWITCH(L.recon, false, return (assemble_t<2, R, MINB>(L, g, list, n, u1, u2, rates, rslot, s)))
  }
  return cudaSuccess;
}
// The split form: the plain pass (own cells and same-level ghosts, 4 CTAs per SM), then the rest
// of the ghosts with the MINB register budget.
template <bool BINS>
cudaError_t assemble_plain(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                           unsigned* rates, int rslot, cudaStream_t s, const int* bins, float* brate,
                           int per_sm = 4) {
  const int g = grid_for(n, per_sm);
  if (L.ndim == 3)
    amrk::amr_assemble_plain<3, BINS><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, rates, rslot, bins, brate);
  else
    amrk::amr_assemble_plain<2, BINS><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.w1, L.w2, rates, rslot, bins, brate);
  return cudaGetLastError();
}
template <int MINB>
cudaError_t assemble_split(const AmrLaunch& L, int per_sm, const int* list, int n, const float4* u1, const float4* u2,
                           unsigned* rates, int rslot, cudaStream_t s) {
  cudaError_t e = assemble_plain<false>(L, list, n, u1, u2, rates, rslot, s, nullptr, nullptr);
  if (e != cudaSuccess || L.nrest == 0) return e;
  const int* rl = L.nrest > 0 ? L.rest : list;
  const int rn = L.nrest > 0 ? L.nrest : n;
  const int g = grid_for(rn, per_sm);
  if (L.ndim == 3) {
    SHZ_RECON_SWITCH(L.recon, false, return (assemble_t<3, R, MINB, false, true>(L, g, rl, rn, u1, u2, rates, rslot, s)))
  } else {
    SHZ_RECON_SWITCH(L.recon, false, return (assemble_t<2, R, MINB, false, true>(L, g, rl, rn, u1, u2, rates, rslot, s)))
  }
  return cudaSuccess;
}
// The split form with its passes side by side: the second (a latency-bound gather of coarse cells
// and restrictions) on the side stream at per_sm CTAs an SM, beside the first (bandwidth-bound) at
// 2 CTAs an SM, so that both are resident at once (the plain pass's 2 x 256 threads x 64 registers
// and the second pass's per_sm x 256 x 128 at most fill one SM's register file).
template <int MINB>
cudaError_t assemble_split_side(const AmrLaunch& L, int per_sm, const int* list, int n, const float4* u1,
                                const float4* u2, unsigned* rates, int rslot, cudaStream_t s) {
  if (!L.side || !L.fork || !L.join || L.nrest == 0) return assemble_split<MINB>(L, per_sm, list, n, u1, u2, rates, rslot, s);
  cudaError_t e = cudaEventRecord(L.fork, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(L.side, L.fork, 0);
  if (e != cudaSuccess) return e;
  const int* rl = L.nrest > 0 ? L.rest : list;
  const int rn = L.nrest > 0 ? L.nrest : n;
  const int g = grid_for(rn, per_sm);
  if (L.ndim == 3) {
    SHZ_RECON_SWITCH(L.recon, false, (e = assemble_t<3, R, MINB, false, true>(L, g, rl, rn, u1, u2, rates, rslot, L.side)))
  } else {
    SHZ_RECON_SWITCH(L.recon, false, (e = assemble_t<2, R, MINB, false, true>(L, g, rl, rn, u1, u2, rates, rslot, L.side)))
  }
  // the join is recorded and waited for whatever the launches returned, so that a capture in
  // progress ends with the side stream joined
  const cudaError_t e2 = assemble_plain<false>(L, list, n, u1, u2, rates, rslot, s, nullptr, nullptr, 2);
  const cudaError_t e3 = cudaEventRecord(L.join, L.side);
  const cudaError_t e4 = cudaStreamWaitEvent(s, L.join, 0);
  return e != cudaSuccess ? e : e2 != cudaSuccess ? e2 : e3 != cudaSuccess ? e3 : e4;
}
}  // namespace

cudaError_t amr_launch_assemble(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                                unsigned* rates, int rslot, cudaStream_t s, const tune::Choice* c) {
  if (n <= 0) return cudaSuccess;
  const int per_sm = c && c->per_sm > 0 ? c->per_sm : 4;
  const int g = grid_for(n, per_sm);
  switch (c ? c->variant : 0) {
    case 1: return assemble_v<2>(L, g, list, n, u1, u2, rates, rslot, s);
    case 2: return assemble_v<3>(L, g, list, n, u1, u2, rates, rslot, s);
    case 3: return assemble_split<2>(L, per_sm, list, n, u1, u2, rates, rslot, s);
    case 4: return assemble_split<3>(L, per_sm, list, n, u1, u2, rates, rslot, s);
    case 5: return assemble_split_side<2>(L, per_sm, list, n, u1, u2, rates, rslot, s);
    case 6: return assemble_split_side<3>(L, per_sm, list, n, u1, u2, rates, rslot, s);
    default: return assemble_v<1>(L, g, list, n, u1, u2, rates, rslot, s);
  }
}

void amr_rest_blocks(const int32_t* bt, int ndim, const int32_t* list, int n, std::vector<int32_t>& out) {
  using amrk::BS;
  out.clear();
  const int S = amrk::BTS;
  auto leaf = [&](int s) { return (bt[(size_t)s * S + 4] & 2) != 0; };
  for (int i = 0; i < n; i++) {
    const int slot = list[i];
    bool rest = !leaf(slot);
    for (int d = 0; d < (ndim == 3 ? 27 : 9) && !rest; d++) {
      const int dir[3] = {d % 3 - 1, (d / 3) % 3 - 1, ndim == 3 ? d / 9 - 1 : 0};
      if (!dir[0] && !dir[1] && !dir[2]) continue;
      int m[3];
      for (int a = 0; a < 3; a++) m[a] = dir[a] < 0 ? -1 : dir[a] > 0 ? BS : 0;
      // ghost_src_any's hops across all but the last out-of-range axis
      int cur = slot;
      for (int hop = 0; hop < ndim; hop++) {
        int out = 0, axis = -1;
        for (int a = 0; a < ndim; a++)
          if (m[a] < 0 || m[a] >= BS) {
            out++;
            if (axis < 0) axis = a;
          }
        if (out <= 1) break;
        const int upper = m[axis] >= BS ? 1 : 0;
        const int nb = bt[(size_t)cur * S + 6 + 2 * axis + upper];
        if (nb >= 0) {
          cur = nb;
          m[axis] += upper ? -BS : BS;
        } else if (nb <= -2) {
          if (-1 - nb == 2) m[axis] = upper ? 2 * BS - 1 - m[axis] : -1 - m[axis];
          else m[axis] = upper ? BS - 1 : 0;
        } else {
          for (int a = 0; a < ndim; a++)
            if (a != axis) m[a] = std::min(std::max(m[a], 0), BS - 1);
        }
      }
      // ghost_src's kind and source block, then plain_src
      int out = 0, axis = 0;
      for (int a = 0; a < ndim; a++)
        if (m[a] < 0 || m[a] >= BS) {
          out++;
          axis = a;
        }
      int src = cur;
      if (out > 1) {
        rest = true;
      } else if (out == 1) {
        const int nb = bt[(size_t)cur * S + 6 + 2 * axis + (m[axis] >= BS ? 1 : 0)];
        if (nb >= 0) src = nb;
        else if (nb == -1) rest = true;
      }
      if (!rest && !leaf(src)) rest = true;
    }
    if (rest) out.push_back(slot);
  }
}

cudaError_t amr_launch_assemble_bins(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                                     const int* bins, unsigned* rates, int rslot, float* brate, cudaStream_t s,
                                     const tune::Choice* c) {
  if (n <= 0) return cudaSuccess;
  const int per_sm = c && c->per_sm > 0 ? c->per_sm : 4;
  const int g = grid_for(n, per_sm);
  if (c && c->variant == 3) {
    // the split form; its second pass walks the whole list, since which neighbours are part way
    // through their step changes from substep to substep
    cudaError_t e = assemble_plain<true>(L, list, n, u1, u2, rates, rslot, s, bins, brate);
    if (e != cudaSuccess) return e;
    if (L.ndim == 3) {
      SHZ_RECON_SWITCH(L.recon, false, return (assemble_t<3, R, 2, true, true>(L, g, list, n, u1, u2, rates, rslot, s, bins, brate)))
    } else {
      SHZ_RECON_SWITCH(L.recon, false, return (assemble_t<2, R, 2, true, true>(L, g, list, n, u1, u2, rates, rslot, s, bins, brate)))
    }
    return cudaSuccess;
  }
  if (L.ndim == 3) {
    SHZ_RECON_SWITCH(L.recon, false, return (assemble_t<3, R, 2, true>(L, g, list, n, u1, u2, rates, rslot, s, bins, brate)))
  } else {
    SHZ_RECON_SWITCH(L.recon, false, return (assemble_t<2, R, 2, true>(L, g, list, n, u1, u2, rates, rslot, s, bins, brate)))
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
__global__ void clock_multi_kernel(DevClock* __restrict__ clks, unsigned* __restrict__ rates, int rslot, int ngrids,
                                   int cycle) {
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
    else dt = fmin(dt, rem / cycle);
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

cudaError_t launch_clock_multi(DevClock* clks, unsigned* rates, int rslot, int ngrids, cudaStream_t s, int cycle) {
  if (ngrids <= 0) return cudaSuccess;
  clock_multi_kernel<<<(ngrids + 127) / 128, 128, 0, s>>>(clks, rates, rslot, ngrids, cycle < 1 ? 1 : cycle);
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

cudaError_t amr_launch_diag_ext(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                                double* part, double* out, cudaStream_t s) {
  const int g = amr_diag_blocks(n);
  if (L.ndim == 3) amrk::amr_diag_ext<3><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, part);
  else amrk::amr_diag_ext<2><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, part);
  dext::final_kernel<<<1, 32, 0, s>>>(part, g, out);
  return cudaGetLastError();
}

cudaError_t amr_launch_ghost_map(const AmrLaunch& L, int slot, int* out, cudaStream_t s) {
  if (L.ndim == 3) amrk::amr_ghost_map<3><<<32, 256, 0, s>>>(L.bt, slot, out);
  else amrk::amr_ghost_map<2><<<2, 256, 0, s>>>(L.bt, slot, out);
  return cudaGetLastError();
}

}  // namespace shz
