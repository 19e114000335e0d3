// Host entry points of the uniform-grid kernels (sweep.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

#include "hydro_math.cuh"

namespace shz {

constexpr int DIAG_VALUES = 9;  // mass, momentum x3, e_kin, e_int, e_tot, floored, max Mach

// tz: planes a CTA marches along z (3D; 0 for the default). Every tz gives the same state.
constexpr int SWEEP_TZ_DEFAULT = 64;
cudaError_t launch_sweep(const KParams& P, int ndim, int recon, bool isen, const float4* u1, const float4* u2, float4* o1,
                         float4* o2, const DevClock* clk, unsigned* rate_out, cudaStream_t s, int tz = 0);
cudaError_t launch_rate(const KParams& P, const float4* u1, const float4* u2, size_t ncell, unsigned* out, cudaStream_t s);
cudaError_t launch_clock(DevClock* clk, unsigned* rates, int slot, cudaStream_t s);
int diag_blocks(size_t ncell);
cudaError_t launch_diag(const KParams& P, const float4* u1, const float4* u2, size_t ncell, double* part, double* out,
                        cudaStream_t s);
size_t sweep_smem_bytes(int ndim, int recon);
int sweep_min_cells(int recon);

}  // namespace shz
