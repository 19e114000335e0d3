// The launch-shape autotuner of the block and sweep kernels.
//
// Each tunable kernel has a small set of compiled variants and runtime launch shapes. The first
// time a driver runs a kernel for a key (kernel, ndim, reconstruction, isentropic, size class),
// it times every candidate in place, on the step's own data, inside one real step: every
// tunable kernel here reads one buffer and writes another (and folds a maximum with atomicMax),
// so running it once or five times leaves the same result. The fastest candidate is kept in a
// process-wide table and used from then on, including in the CUDA graphs the drivers capture.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <vector>

namespace shz {
namespace tune {

enum Kernel : int {
  K_UNIFORM_SWEEP = 0,  // tz: planes a CTA marches along z (3D); 2D (>= 512 a side): rows along y
  K_AMR_ASSEMBLE = 1,   // variant: register budget (CTAs per SM the compiler plans for); per_sm: grid
  K_AMR_SWEEP = 2,      // per_sm: grid
  K_AMR_FINE_FLUX = 3,  // per_sm: grid
  K_AMR_ASSEMBLE_BINS = 4,  // the per-block-timestep substeps' assemble: variant 1 one pass, 3 split
  K_COUNT = 5
};

struct Key {
  int kernel, ndim, recon, isen, size_class;
  bool operator<(const Key& o) const;
};

struct Choice {
  int variant = 0;
  int per_sm = 0;  // 0: the kernel's default
  int tz = 0;      // 0: the kernel's default
};

struct Entry {
  Key key;
  Choice choice;
  float ms = 0.f;          // the chosen candidate's mean time
  float default_ms = 0.f;  // the default candidate's
  int candidates = 0;
};

// Process-wide switch (on by default). Off: every launch takes the kernel's default shape.
bool enabled();
void set_enabled(bool on);
void reset();

// floor(log2(units)): the size class of a key.
int size_class(long long units);

// The tuned choice for `k`, if any.
bool lookup(const Key& k, Choice* out);

// A choice pinned for every key of one kernel (a check that every candidate gives the same
// state, or a fixed shape): the drivers use it instead of tuning. pin(kernel, nullptr) unpins.
void pin(int kernel, const Choice* c);
bool pinned(int kernel, Choice* out);

// Whether `k` still needs tuning (the tuner is on and no choice is stored).
bool needs(const Key& k);

// Time each candidate's launch functor on stream s (one warm-up launch, then `reps` timed
// launches with CUDA events), store the fastest for k and return it; candidates[0] is the
// default. On a launch error the error is returned and nothing is stored.
cudaError_t choose(const Key& k, const std::vector<Choice>& candidates,
                   const std::function<cudaError_t(const Choice&)>& launch, cudaStream_t s, int reps, Choice* out);

std::vector<Entry> entries();

}  // namespace tune
}  // namespace shz
