// The diagnostics channels beyond the conservation totals (hydro/diagnostics.wgsl channels 10-22,
// src/sim.ts:1808 DIAG_OPS; read back as Diagnostics.ranges and .com, src/sim.ts:1650-1667):
// the smallest and largest density, temperature, scalar, pressure and speed over the cells, and
// the centre of mass's numerators (sum rho dV x). Shared by the uniform grid (sweep.cu) and the
// block grid (amr_kernels.cu); float64, fixed reduction order, compensated sums.
#pragma once
#include <cuda_runtime.h>

#include "hydro_math.cuh"

namespace shz {
namespace dext {

// Values per block and in the result: min of the five fields, max of the five, three sums.
constexpr int N = 13;

struct Comp {
  double s = 0.0, c = 0.0;
  __device__ void add(double x) {
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  __device__ double value() const { return s + c; }
};

struct Ext {
  double mn[5], mx[5];
  Comp com[3];
  __device__ void init() {
#pragma unroll
    for (int i = 0; i < 5; i++) {
      mn[i] = __longlong_as_double(0x7ff0000000000000LL);   // +inf
      mx[i] = __longlong_as_double((long long)0xfff0000000000000ULL);  // -inf
    }
  }
  // One cell of volume dv at (x, y, z) from the box centre, as diagnostics.wgsl:13-97 forms it for
  // an ideal gas: rho floored, p = (gamma - 1) e_int floored, T = (gamma - 1) e_int / rho, the
  // scalar rho s / rho, the speed |v|.
  __device__ void cell(const float4 a, const float4 b, const KParams& P, double dv, double x, double y, double z) {
    const double rho = fmax((double)a.x, (double)P.rho_floor);
    const double eint = b.y;
    const double p = fmax((double)P.gm1 * eint, (double)P.p_floor);
    const double T = (double)P.gm1 * eint / rho;
    const double s = (double)b.z / rho;
    const double vx = a.y / rho, vy = a.z / rho, vz = a.w / rho;
    const double f[5] = {rho, T, s, p, sqrt(vx * vx + vy * vy + vz * vz)};
#pragma unroll
    for (int i = 0; i < 5; i++) {
      mn[i] = fmin(mn[i], f[i]);
      mx[i] = fmax(mx[i], f[i]);
    }
    com[0].add(rho * dv * x);
    com[1].add(rho * dv * y);
    com[2].add(rho * dv * z);
  }
};

__device__ __forceinline__ double combine(int i, double a, double b) {
  return i < 5 ? fmin(a, b) : (i < 10 ? fmax(a, b) : a + b);
}

// The block's N values into out (thread 0 writes): each warp's lanes, then the warps, in order.
__device__ __forceinline__ void block_reduce(const Ext& e, double* __restrict__ out) {
  __shared__ double sh[32][N];
  double v[N];
#pragma unroll
  for (int i = 0; i < 5; i++) {
    v[i] = e.mn[i];
    v[5 + i] = e.mx[i];
  }
#pragma unroll
  for (int i = 0; i < 3; i++) v[10 + i] = e.com[i].value();
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int i = 0; i < N; i++) v[i] = combine(i, v[i], __shfl_down_sync(0xffffffffu, v[i], off));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < N; i++) sh[warp][i] = v[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int i = 0; i < N; i++) {
      Comp c;
      double m = sh[0][i];
      for (int w = 0; w < nw; w++) {
        if (i >= 10) c.add(sh[w][i]);
        else if (w > 0) m = combine(i, m, sh[w][i]);
      }
      out[i] = i >= 10 ? c.value() : m;
    }
  }
}

// The blocks' values combined in block order, one thread per value (internal linkage: each file
// that launches it has its own copy).
static __global__ void final_kernel(const double* __restrict__ part, int nblocks, double* __restrict__ out) {
  const int i = threadIdx.x;
  if (i >= N) return;
  Comp c;
  double m = part[i];
  for (int b = 0; b < nblocks; b++) {
    const double x = part[(size_t)b * N + i];
    if (i >= 10) c.add(x);
    else if (b > 0) m = combine(i, m, x);
  }
  out[i] = i >= 10 ? c.value() : m;
}

}  // namespace dext
}  // namespace shz
