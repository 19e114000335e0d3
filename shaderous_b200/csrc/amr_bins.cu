// Per-block timesteps on the adaptive grid (amr/bins_*.wgsl, amr/mid_on.wgsl): the bins of a cycle
// and the clock's substep bookkeeping. The other passes of a substep take the bin table: the
// assemble (amr_kernels.cu), the fused sweep with its neighbour-flux pass and deposits
// (amr_sweep.cu), or the two passes (amr_twopass.cu).
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
