// Host entry points of the adaptive-grid passes (amr_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "hydro_math.cuh"
#include "tune.h"

namespace shz {

// What every pass needs: the scheme, the per-grid parameters and clocks, the block table and
// the two derived atlases. Word 26 of a block's table row names its grid; a grid's KParams hold
// its level-0 cell size in dx and its root blocks per side in n[0].
struct AmrLaunch {
  int ndim;
  int recon;
  bool isen;
  const KParams* gp;   // device, per grid
  const int* bt;
  float4* w1;   // primitives with ghosts, 20^ndim texels per slot
  float4* w2;
  float4* p1;   // half steps, 18^ndim texels per slot (the two-pass step only; else null)
  float4* p2;
  // Fine-flux buffer of the fused sweep: 2 float4 per face cell (16^(ndim-1) cells) per matched
  // face; a leaf's row holds its first entry in word 27 (-1: none).
  float4* fbuf = nullptr;
  // Device error word the kernels set when a bounded wait runs out (tma::ERR_*); read and cleared
  // by the host.
  int* err = nullptr;
  // The assemble forms every coarse ghost's prolongation itself, as the reference does (the two-pass
  // mode), instead of from its per-block table of coarse cells; the numbers are the same.
  bool per_texel = false;
  // Per-block timesteps, for the fused sweep, its neighbour-flux pass and the deposits: the bin
  // table ([0] the substep, [1 + slot] the bin; null: one timestep) and, per slot, the first entry
  // of its faces' fluxes in fbuf for this substep (-1: none).
  const int* bins = nullptr;
  const int* fbase = nullptr;
  // The split assemble's second pass walks these blocks only (amr_rest_blocks over the list the
  // assemble is given); nrest < 0: every block of that list.
  const int* rest = nullptr;
  int nrest = -1;
  // The owner's second stream and two events (all null: none): the split assemble's two passes
  // write disjoint texels and read only the state, so variants 5 and 6 run the second on `side`
  // beside the first (fork and join order it against the owner's stream, graph capture included).
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

// The blocks of `list` (n slots; bt the host copy of the block table, 32 ints a row) with a ghost
// texel whose source is not a cell of a same-level leaf: a coarser leaf beyond a face, or a
// refined neighbour, whose cells are restricted; every parent. Each of the 26 (2D: 8) neighbour
// directions is resolved as the assemble's ghost_src_any resolves every texel in it (the hops
// and the final face give the same blocks wherever the texel lies in that direction's region).
void amr_rest_blocks(const int32_t* bt, int ndim, const int32_t* list, int n, std::vector<int32_t>& out);

// rates: two 32-bit maxima per grid; the assemble folds the leaves' rate / dx into slot rslot.
// c: the autotuner's choice (null: the default shape), as for the fine-flux pass and the sweep.
cudaError_t amr_launch_assemble(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                                unsigned* rates, int rslot, cudaStream_t s, const tune::Choice* c = nullptr);
// The clocks of `ngrids` grids at once (one thread each): dt from each grid's rate slot. With
// cycle > 1 (per-block timesteps) the step is repeated for a cycle of that many substeps, and is
// kept short enough for the cycle to end by the stop time.
cudaError_t launch_clock_multi(DevClock* clks, unsigned* rates, int rslot, int ngrids, cudaStream_t s, int cycle = 1);
// The two passes (amr_twopass.cu); bins: the per-block timesteps' bin table (null: one timestep).
// With bins the update writes in place: o1, o2 are u1, u2.
cudaError_t amr_launch_predict(const AmrLaunch& L, const int* list, int n, const DevClock* clks, cudaStream_t s,
                               const int* bins = nullptr);
cudaError_t amr_launch_update(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, float4* o1,
                              float4* o2, const DevClock* clks, cudaStream_t s, const int* bins = nullptr);
// Per-block timesteps (amr_bins.cu).
// The assemble of the blocks in list for a substep: as amr_launch_assemble (coarse ghosts from the
// block's tables, or each formed by itself in the two-pass form), with the ghosts of neighbours
// part way through a longer step taken from their half-step atlas; each leaf's own rate / dx also
// goes to brate[slot] (if not null).
// c: the launch shape (null: the one-pass kernel, 4 CTAs per SM; variant 3: the split form).
cudaError_t amr_launch_assemble_bins(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                                     const int* bins, unsigned* rates, int rslot, float* brate, cudaStream_t s,
                                     const tune::Choice* c = nullptr);
// The same with the tuned shape (kernel K_AMR_ASSEMBLE_BINS), tuned in place on its first call for
// a key (these substep launches are eager); *extra grows by the kernels launched beyond the one
// the caller counts (the split form's second pass, the tuning launches).
cudaError_t amr_assemble_bins_tuned(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                                    const int* bins, unsigned* rates, int rslot, float* brate, cudaStream_t s,
                                    long long* extra);
// The bins of a cycle over the blocks in list (all of them): the first guess from each leaf's rate
// and the clock's dt into `a`, then the dilation sweep into `b` and `sweeps` (odd) relaxation
// sweeps alternating b -> a, a -> b, ..., so that the result is in `a`.
cudaError_t amr_launch_bins(const AmrLaunch& L, const int* list, int n, const float* brate, const DevClock* clk,
                            float cfl, int kmax, int sweeps, int* a, int* b, cudaStream_t s);
// Substep s of a cycle begins: the bin table's substep word, and the clock banks the substep.
cudaError_t amr_launch_bins_tick(DevClock* clk, int* bins, int s, cudaStream_t st);
// The mean fine fluxes of the matched faces listed in flist (leaf slot, face, buffer entry per
// face), into L.fbuf; before the sweep.
cudaError_t amr_launch_fine_flux(const AmrLaunch& L, const int* flist, int nf, const DevClock* clks, cudaStream_t s,
                                 const tune::Choice* c = nullptr);
// Predict, fluxes and update of every leaf in one pass over the primitive atlas (no half-step
// atlas), standing for predict + update.
cudaError_t amr_launch_sweep(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, float4* o1,
                             float4* o2, const DevClock* clks, cudaStream_t s, const tune::Choice* c = nullptr);
// Per-block timesteps, fused form: the leaves in list half way through their step beside a faster
// neighbour take that neighbour's second-step fluxes from fbuf, in place (amr/update.wgsl deposit).
cudaError_t amr_launch_deposit(const AmrLaunch& L, const int* list, int n, float4* u1, float4* u2, const DevClock* clks,
                               cudaStream_t s);
cudaError_t amr_launch_flag(const AmrLaunch& L, const int* list, int n, float* flags, cudaStream_t s);
cudaError_t amr_launch_regrid(const AmrLaunch& L, const int* rg, const int* list, int n, const float4* u1,
                              const float4* u2, float4* o1, float4* o2, cudaStream_t s);
int amr_diag_blocks(int n);
cudaError_t amr_launch_diag(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, double* part,
                            double* out, cudaStream_t s);
// The extended diagnostics channels (diag_ext.cuh, 13 values) over the leaves in list; part holds
// amr_diag_blocks(n) x 13 doubles.
cudaError_t amr_launch_diag_ext(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                                double* part, double* out, cudaStream_t s);
cudaError_t amr_launch_ghost_map(const AmrLaunch& L, int slot, int* out, cudaStream_t s);

}  // namespace shz

namespace shz {

// Launch with the autotuner's shape for the key; when the key has none yet and `tune_now` is set
// (an eager step, not a graph capture), time every candidate in place and keep the fastest.
// *launches grows by the kernels launched.
tune::Key amr_tune_key(int kernel, const AmrLaunch& L, long long units);
cudaError_t amr_assemble_tuned(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2,
                               unsigned* rates, int rslot, cudaStream_t s, bool tune_now, long long* launches);
cudaError_t amr_fine_flux_tuned(const AmrLaunch& L, const int* flist, int nf, const DevClock* clks, cudaStream_t s,
                                bool tune_now, long long* launches);
cudaError_t amr_sweep_tuned(const AmrLaunch& L, const int* list, int n, const float4* u1, const float4* u2, float4* o1,
                            float4* o2, const DevClock* clks, cudaStream_t s, bool tune_now, long long* launches);
// Whether a step over n leaves (nf matched faces) would tune anything.
bool amr_step_wants_tuning(const AmrLaunch& L, int n_assembled, int n_leaves, int nf);

}  // namespace shz
