// The launch-shape autotuner: a process-wide table of the fastest candidate per key.
#include "tune.h"

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>

#include "../../include/shaderous_b200.h"

namespace shz {
namespace tune {

namespace {
std::mutex g_mu;
std::map<Key, Entry> g_table;
std::atomic<bool> g_on{true};
}  // namespace

bool Key::operator<(const Key& o) const {
  if (kernel != o.kernel) return kernel < o.kernel;
  if (ndim != o.ndim) return ndim < o.ndim;
  if (recon != o.recon) return recon < o.recon;
  if (isen != o.isen) return isen < o.isen;
  return size_class < o.size_class;
}

bool enabled() { return g_on.load(); }
void set_enabled(bool on) { g_on.store(on); }

void reset() {
  std::lock_guard<std::mutex> lk(g_mu);
  g_table.clear();
}

int size_class(long long units) {
  int c = 0;
  while (units > 1) {
    units >>= 1;
    c++;
  }
  return c;
}

namespace {
Choice g_pin[K_COUNT];
bool g_pinned[K_COUNT] = {};
}  // namespace

void pin(int kernel, const Choice* c) {
  if (kernel < 0 || kernel >= K_COUNT) return;
  std::lock_guard<std::mutex> lk(g_mu);
  g_pinned[kernel] = c != nullptr;
  if (c) g_pin[kernel] = *c;
}

bool pinned(int kernel, Choice* out) {
  if (kernel < 0 || kernel >= K_COUNT) return false;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_pinned[kernel]) return false;
  *out = g_pin[kernel];
  return true;
}

bool lookup(const Key& k, Choice* out) {
  if (!enabled()) return false;
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_table.find(k);
  if (it == g_table.end()) return false;
  *out = it->second.choice;
  return true;
}

bool needs(const Key& k) {
  if (!enabled()) return false;
  std::lock_guard<std::mutex> lk(g_mu);
  return g_table.find(k) == g_table.end();
}

cudaError_t choose(const Key& k, const std::vector<Choice>& candidates,
                   const std::function<cudaError_t(const Choice&)>& launch, cudaStream_t s, int reps, Choice* out) {
  if (candidates.empty()) return cudaErrorInvalidValue;
  cudaEvent_t e0, e1;
  cudaError_t e = cudaEventCreate(&e0);
  if (e != cudaSuccess) return e;
  e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cudaEventDestroy(e0);
    return e;
  }
  std::vector<float> ms(candidates.size(), 0.f);
  for (size_t i = 0; i < candidates.size() && e == cudaSuccess; i++) {
    e = launch(candidates[i]);  // warm-up (and the first application of the step)
    if (e == cudaSuccess) e = cudaEventRecord(e0, s);
    for (int r = 0; r < reps && e == cudaSuccess; r++) e = launch(candidates[i]);
    if (e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms[i], e0, e1);
    ms[i] /= (float)std::max(reps, 1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return e;
  const size_t best = (size_t)(std::min_element(ms.begin(), ms.end()) - ms.begin());
  Entry en;
  en.key = k;
  en.choice = candidates[best];
  en.ms = ms[best];
  en.default_ms = ms[0];
  en.candidates = (int)candidates.size();
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_table[k] = en;
  }
  *out = candidates[best];
  return cudaSuccess;
}

std::vector<Entry> entries() {
  std::lock_guard<std::mutex> lk(g_mu);
  std::vector<Entry> v;
  for (const auto& kv : g_table) v.push_back(kv.second);
  return v;
}

}  // namespace tune
}  // namespace shz

extern "C" {

int shz_tune_enable(int32_t on) {
  shz::tune::set_enabled(on != 0);
  return 0;
}

void shz_tune_reset(void) { shz::tune::reset(); }

int shz_tune_pin(int32_t kernel, int32_t variant, int32_t per_sm) {
  if (kernel < 0 || kernel >= shz::tune::K_COUNT) return SHZ_E_CONFIG;
  if (variant < 0) {
    shz::tune::pin(kernel, nullptr);
    return 0;
  }
  // the variants each kernel compiles (the assemble's 0-6, the substeps' assemble's 1 and 3; the
  // others' 0)
  const bool ok = kernel == shz::tune::K_AMR_ASSEMBLE        ? variant <= 6
                  : kernel == shz::tune::K_AMR_ASSEMBLE_BINS ? (variant == 1 || variant == 3)
                                                             : variant == 0;
  // (the uniform sweep's knob is its depth, given in per_sm)
  const int most = kernel == shz::tune::K_UNIFORM_SWEEP ? 1024 : 32;
  if (!ok || per_sm < 0 || per_sm > most) return SHZ_E_CONFIG;
  shz::tune::Choice c;
  c.variant = variant;
  if (kernel == shz::tune::K_UNIFORM_SWEEP) c.tz = per_sm;
  else c.per_sm = per_sm;
  shz::tune::pin(kernel, &c);
  return 0;
}

int shz_tune_entries(shz_tune_entry* out, int32_t max, int32_t* n) {
  if (!n || max < 0 || (max > 0 && !out)) return SHZ_E_CONFIG;
  const std::vector<shz::tune::Entry> v = shz::tune::entries();
  *n = (int32_t)v.size();
  for (int i = 0; i < (int)v.size() && i < max; i++) {
    const auto& e = v[i];
    shz_tune_entry& o = out[i];
    o.kernel = e.key.kernel;
    o.ndim = e.key.ndim;
    o.recon = e.key.recon;
    o.isentropic = e.key.isen;
    o.size_class = e.key.size_class;
    o.variant = e.choice.variant;
    o.per_sm = e.choice.per_sm;
    o.tz = e.choice.tz;
    o.candidates = e.candidates;
    o.ms = e.ms;
    o.default_ms = e.default_ms;
  }
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// A check of the kernels' bounded-wait path, without any fault: one CTA waits on an mbarrier
// phase that nothing completes, with a short limit, and must come back with the timeout code in
// its error word, as a copy that never lands would make the sweeps do.
#include "tma.cuh"

namespace {
__global__ void wait_timeout_kernel(int* err, uint32_t limit) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    shz::tma::mbar_init(&bar, 1);
    shz::tma::fence_mbar_init();
  }
  __syncthreads();
  // phase 0 never completes: no thread arrives on it
  const bool ok = shz::tma::mbar_wait(&bar, 0u, limit);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicExch(err, shz::tma::ERR_TMA_TIMEOUT);
    return;
  }
  if (threadIdx.x == 0) atomicExch(err, -1);  // (cannot happen: the phase has no arrivals)
}
}  // namespace

extern "C" int shz_selftest_wait_timeout(int32_t device, int32_t* code) {
  if (!code) return SHZ_E_CONFIG;
  int prev = -1;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return SHZ_E_NODEV;
  int* d = nullptr;
  int rc = SHZ_OK;
  if (cudaMalloc(&d, sizeof(int)) != cudaSuccess || cudaMemset(d, 0, sizeof(int)) != cudaSuccess) rc = SHZ_E_CUDA;
  if (rc == SHZ_OK) {
    wait_timeout_kernel<<<1, 64>>>(d, 1000u);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = SHZ_E_CUDA;
  }
  int h = 0;
  if (rc == SHZ_OK && cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) rc = SHZ_E_CUDA;
  if (d) cudaFree(d);
  if (prev >= 0) cudaSetDevice(prev);
  *code = h;
  return rc;
}
