// Host entry points of the adaptive-grid passes (amr_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "hydro_math.cuh"

namespace shz {

// What every pass needs: hydro parameters, the block table and the two derived atlases.
struct AmrLaunch {
  KParams P;
  int ndim;
  int recon;
  bool isen;
  int nr;       // root blocks per side
  double dx0;   // cell size at level 0
  const int* bt;
  float4* w1;   // primitives with ghosts, 20^ndim texels per slot
  float4* w2;
  float4* p1;   // half steps, 18^ndim texels per slot
  float4* p2;
};

cudaError_t amr_launch_assemble(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                                unsigned* rate_out, cudaStream_t s);
cudaError_t amr_launch_predict(const AmrLaunch& L, const int* list, int n, const DevClock* clk, cudaStream_t s);
cudaError_t amr_launch_update(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, float4* o1,
                              float4* o2, const DevClock* clk, cudaStream_t s);
cudaError_t amr_launch_flag(const AmrLaunch& L, const int* list, int n, float* flags, cudaStream_t s);
cudaError_t amr_launch_regrid(const AmrLaunch& L, const int* rg, const int* list, int n, const float4* u1,
                              const float4* u2, float4* o1, float4* o2, cudaStream_t s);
int amr_diag_blocks(int n);
cudaError_t amr_launch_diag(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, double* part,
                            double* out, cudaStream_t s);
cudaError_t amr_launch_ghost_map(const AmrLaunch& L, int slot, int* out, cudaStream_t s);

}  // namespace shz
