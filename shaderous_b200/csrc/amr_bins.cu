// Per-block timesteps on the adaptive grid (amr/bins_*.wgsl, amr/mid_on.wgsl): the assemble of a
// substep, the bins of a cycle and the clock's substep bookkeeping. The predict and update passes
// of a substep are the two passes' own (amr_twopass.cu), given the bin table.
//
// Time advances in cycles of 2^K substeps of the clock's dt, the step of the fastest block. At the
// start of a cycle every block steps; in between, the blocks of bin k start a step on the
// substeps that are multiples of 2^k. A block part way through its step has already stored the
// state of its end; its neighbours that start a step meanwhile take its half-step prediction,
// kept from its own start, for their ghosts (the scheme's estimate of the state at that time).
// Bins are set once per cycle from each leaf's own signal rate, then relaxed until face
// neighbours are at most one bin apart, no block is slower than a coarser neighbour, and a
// parent is as fast as its fastest child (amr/bins_init.wgsl, amr/bins_relax.wgsl).
#include <cuda_runtime.h>

#include "amr_device.cuh"

namespace shz {
namespace amrk {

// from_coarse (amr_device.cuh) for a coarse leaf part way through its step: the coarse cell and
// its neighbours along the axes from its half-step atlas (which covers its first ghost layer), no
// boundary mapping needed (amr/assemble.wgsl:59-66).
template <int DIM, int R>
__device__ __forceinline__ Cons from_coarse_mid(const KParams& P, const int* __restrict__ bt, const float4* __restrict__ p1,
                                                const float4* __restrict__ p2, int nr, int slot, const int* l, int cs) {
  const int nc = nr * BS << bt_at(bt, cs, 0);
  int lc[3], par[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int gf = a < DIM ? bt_at(bt, slot, 1 + a) * BS + l[a] : 0;
    int gc = gf >> 1;
    gc = ((gc % nc) + nc) % nc;
    lc[a] = a < DIM ? gc - bt_at(bt, cs, 1 + a) * BS : 0;
    par[a] = a < DIM ? (gf & 1) : 0;
  }
  const Cons uc = mid_cons<DIM>(P, p1, p2, cs, lc);
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
  const Slopes sl = prolong_slopes<DIM, R>(uc, m, ok, p, ok, P.rho_floor);
  return prolong_child(uc, sl, par);
}

// The assemble of a substep (amr/assemble.wgsl:78-154 with <bins> and <mid>): every texel of each
// listed block's primitive atlas from its source, where a source leaf part way through its step
// gives its half-step state. The leaves' rate / dx goes to the grid's maximum and to the block's
// own entry of brate.
template <int DIM, int R>
__global__ void __launch_bounds__(NT) amr_assemble_bins(const KParams* __restrict__ gp, const int* __restrict__ bt,
                                                        const int* __restrict__ list, int n, const float4* __restrict__ u1,
                                                        const float4* __restrict__ u2, const float4* __restrict__ p1,
                                                        const float4* __restrict__ p2, const int* __restrict__ bins,
                                                        float4* __restrict__ w1, float4* __restrict__ w2,
                                                        unsigned* __restrict__ rates, int rslot, float* __restrict__ brate) {
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
        u = mid_block(bt, bins, s.slot) ? mid_cons<DIM>(P, p1, p2, s.slot, s.l) : u_at<DIM>(bt, u1, u2, s.slot, s.l);
      } else if (mid_block(bt, bins, s.slot)) {
        u = from_coarse_mid<DIM, R>(P, bt, p1, p2, nr, s.from, s.l, s.slot);
      } else {
        u = from_coarse<DIM, R>(bt, u1, u2, nr, s.from, s.l, s.slot, P.rho_floor);
      }
      u.a.y *= s.flip[0];
      u.a.z *= s.flip[1];
      u.a.w *= s.flip[2];
      float w[7];
      prim_from_cons(u.a, u.b, P, 1.f, 1.f, 1.f, w);
      const size_t o = (size_t)slot * BG<DIM>::WN + t;
      w1[o] = make_float4(w[0], w[1], w[2], w[3]);
      w2[o] = make_float4(w[4], w[5], w[6], 0.f);
      bool inside = leaf;
#pragma unroll
      for (int q = 0; q < DIM; q++) inside = inside && l[q] >= 0 && l[q] < BS;
      if (inside) rmax = fmaxf(rmax, rate_guard_f(fabsf(w[1]) + fabsf(w[2]) + fabsf(w[3]) + P.signal * w[6]) * inv_dx);
    }
    const float m = block_max(rmax, sRed);
    if (threadIdx.x == 0 && leaf) {
      atomicMax(rates + 2 * g + rslot, __float_as_uint(m));
      if (brate) brate[slot] = m;
    }
  }
}

// First guess of every block's bin at the start of a cycle (amr/bins_init.wgsl): the largest
// power of two of the clock's dt that the leaf's own rate allows, k = floor(log2(dtb / dt))
// clamped to [0, kmax], with dtb = cfl / rate in float32. The floor of the logarithm is taken
// exactly, as the largest k with 2^k <= dtb / dt, from correctly rounded divisions. Parents and
// held steps start at kmax.
__global__ void bins_init_kernel(const int* __restrict__ bt, const int* __restrict__ list, int n,
                                 const float* __restrict__ brate, const DevClock* __restrict__ clk, float cfl, int kmax,
                                 int* __restrict__ kout) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int slot = __ldg(list + i);
  int k = kmax;
  const float dt = (float)clk->dt;
  if (leaf_of(bt, slot) && dt > 0.f) {
    const float dtb = __fdiv_rn(cfl, fmaxf(brate[slot], 1e-30f));
    const float x = __fdiv_rn(dtb, dt);
    k = 0;
    while (k < kmax && x >= (float)(2 << k)) k++;
  }
  kout[1 + slot] = k;
}

// One sweep of the bins toward the rules (amr/bins_relax.wgsl; face neighbours only, as for the
// gas alone): a leaf no slower than one bin above a same-level neighbour (the dilation sweep: no
// slower than it) and than a coarser neighbour; a parent the fastest of its children.
__global__ void bins_relax_kernel(const int* __restrict__ bt, const int* __restrict__ list, int n, int nfaces, int kmax,
                                  int dilate, const int* __restrict__ kin, int* __restrict__ kout) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int slot = __ldg(list + i);
  int k = kin[1 + slot];
  if (!leaf_of(bt, slot)) {
    k = kmax;
    for (int ch = 0; ch < 8; ch++) {
      const int c = bt_at(bt, slot, 12 + ch);
      if (c >= 0) k = min(k, kin[1 + c]);
    }
  } else {
    for (int f = 0; f < nfaces; f++) {
      const int nb = bt_at(bt, slot, 6 + f);
      if (nb >= 0 && nb != slot) k = min(k, kin[1 + nb] + (dilate ? 0 : 1));
      else if (nb == -1) k = min(k, kin[1 + bt_at(bt, slot, 20 + f)]);
    }
  }
  kout[1 + slot] = k;
}

// A substep after the first (amr/bins_tick.wgsl): the substep word of the bin table, and the clock
// banks the substep's dt (held cycles bank nothing).
__global__ void bins_tick_kernel(DevClock* __restrict__ clk, int* __restrict__ bins, int s) {
  bins[0] = s;
  if (s > 0 && !clk->held && clk->dt > 0.0) {
    clk->t += clk->dt;
    clk->steps += 1;
    clk->last_dt = clk->dt;
  }
}

}  // namespace amrk

cudaError_t amr_launch_assemble_bins(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                                     const int* bins, unsigned* rates, int rslot, float* brate, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int g = grid_for(n, 4);
  if (L.ndim == 3) {
    SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_assemble_bins<3, R><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.p1, L.p2, bins, L.w1, L.w2, rates, rslot, brate)))
  } else {
    SHZ_RECON_SWITCH(L.recon, false, (amrk::amr_assemble_bins<2, R><<<g, amrk::NT, 0, s>>>(L.gp, L.bt, list, n, u1, u2, L.p1, L.p2, bins, L.w1, L.w2, rates, rslot, brate)))
  }
  return cudaGetLastError();
}

cudaError_t amr_launch_bins(const AmrLaunch& L, const int* list, int n, const float* brate, const DevClock* clk,
                            float cfl, int kmax, int sweeps, int* a, int* b, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int g = (n + 127) / 128;
  const int nf = 2 * L.ndim;
  amrk::bins_init_kernel<<<g, 128, 0, s>>>(L.bt, list, n, brate, clk, cfl, kmax, a);
  amrk::bins_relax_kernel<<<g, 128, 0, s>>>(L.bt, list, n, nf, kmax, 1, a, b);
  for (int i = 0; i < sweeps; i++) {
    const bool to_a = (i % 2) == 0;
    amrk::bins_relax_kernel<<<g, 128, 0, s>>>(L.bt, list, n, nf, kmax, 0, to_a ? b : a, to_a ? a : b);
  }
  return cudaGetLastError();
}

cudaError_t amr_launch_bins_tick(DevClock* clk, int* bins, int s, cudaStream_t st) {
  amrk::bins_tick_kernel<<<1, 1, 0, st>>>(clk, bins, s);
  return cudaGetLastError();
}

}  // namespace shz
