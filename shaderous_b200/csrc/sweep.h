// Host entry points of the uniform-grid kernels (sweep.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstddef>

#include <cuda.h>

#include "hydro_math.cuh"

namespace shz {

constexpr int DIAG_VALUES = 9;  // mass, momentum x3, e_kin, e_int, e_tot, floored, max Mach

// A grid's dimensionality from its size: the highest axis with more than one cell.
inline int ndim_of_size(const int n[3]) { return n[2] > 1 ? 3 : (n[1] > 1 ? 2 : 1); }

// Tensor maps of one parity of a 3D state, for the sweep's TMA staging of its planes.
struct SweepMaps {
  CUtensorMap u1, u2;
  int zofs = 0;  // planes of the allocation below the grid's first (halo planes of a slab)
  bool valid = false;
};
// Encode the maps of arrays whose allocations start at base1 / base2 (`planes` planes of nx x ny
// float4, the grid's first at zofs); false if the driver cannot (then the sweep loads per cell).
bool encode_sweep_maps(SweepMaps* m, const float4* base1, const float4* base2, int nx, int ny, int planes, int zofs,
                       int recon);

// tz: planes a CTA marches along z (3D; 0 for the default); in 2D, rows a CTA marches along y (the
// row form), or 0 for the tile form. Every tz gives the same state, with or without maps (the
// staging path and the per-cell loads give the same primitives). err: the kernel's error word (a
// bounded wait for a copy that ran out), or null.
constexpr int SWEEP_TZ_DEFAULT = 64;
cudaError_t launch_sweep(const KParams& P, int ndim, int recon, bool isen, const float4* u1, const float4* u2, float4* o1,
                         float4* o2, const DevClock* clk, unsigned* rate_out, cudaStream_t s, int tz = 0,
                         const SweepMaps* maps = nullptr, int* err = nullptr);
cudaError_t launch_rate(const KParams& P, const float4* u1, const float4* u2, size_t ncell, unsigned* out, cudaStream_t s);
cudaError_t launch_clock(DevClock* clk, unsigned* rates, int slot, cudaStream_t s);
int diag_blocks(size_t ncell);
cudaError_t launch_diag(const KParams& P, const float4* u1, const float4* u2, size_t ncell, double* part, double* out,
                        cudaStream_t s);
// The extended diagnostics channels (diag_ext.cuh, 13 values) of a state; part holds
// diag_blocks(ncell) x 13 doubles.
constexpr int DIAG_EXT_VALUES = 13;
cudaError_t launch_diag_ext(const KParams& P, const float4* u1, const float4* u2, size_t ncell, double* part, double* out,
                            cudaStream_t s);
size_t sweep_smem_bytes(int ndim, int recon);
int sweep_min_cells(int recon);

}  // namespace shz
