// The conservation totals of a caller-owned state, with no device allocation at all.
//
// shz_diagnostics() sums the state of a handle into per-block partials that the handle
// allocated with cudaMalloc. Some callers cannot let a library allocate device memory: a host
// that owns all of its GPU memory in its own pool or fixed arena (a serving process that admits
// work against a fixed HBM budget and must account for every byte), or a binding that is handed
// device buffers owned by another runtime and has no allocator of its own to call. For them,
// shz_totals_noalloc() runs the same two reduction kernels with their partials in a file-scope
// device array instead.
//
// The array, g_totals_scratch, holds SHZ_TOTALS_MAX_BLOCKS rows of SHZ_DIAG_VALUES doubles
// (576 KiB). Every GPU that loads this library holds it until the process exits. One row serves
// SHZ_TOTALS_CELLS_PER_BLOCK cells, so a state of more than
// SHZ_TOTALS_MAX_BLOCKS * SHZ_TOTALS_CELLS_PER_BLOCK = 134,217,728 cells (512^3) is refused.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>
#include <utility>

#include "../../include/shaderous_b200.h"
#include "hydro_math.cuh"
#include "sweep.h"

namespace shz {
// The reduction kernels of the handle's diagnostics (sweep.cu), launched here with another
// scratch buffer; their code is shared, not copied.
__global__ void diag_partial_kernel(const KParams P, const float4* __restrict__ u1, const float4* __restrict__ u2,
                                    size_t ncell, double* __restrict__ part);
__global__ void diag_final_kernel(const double* __restrict__ part, int nblocks, double* __restrict__ out);
}  // namespace shz

namespace {

static __device__ __align__(256) double g_totals_scratch[SHZ_TOTALS_MAX_BLOCKS * SHZ_DIAG_VALUES];

constexpr int kMaxDevices = 64;

// The array's device address as looked up on a device, with the unique id of the context it was
// looked up in. A device reset (cudaDeviceReset) or any other teardown of the context reloads the
// module at another address under a context with a new id, so the address is looked up again
// then instead of being reused.
struct ScratchAddr {
  unsigned long long ctx_id = 0;
  double* addr = nullptr;
};
std::mutex g_mu;
ScratchAddr g_addr[kMaxDevices];

// The failing call's message, per calling thread: a failure on one thread neither replaces nor
// frees the text another thread is reading.
thread_local std::string t_msg;

int refuse(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  t_msg = buf;
  return code;
}

// The id of the current context (cuCtxGetCurrent + cuCtxGetId through the runtime's driver entry
// points, so the library needs no link to libcuda). False when either is unavailable.
bool current_context_id(unsigned long long* id) {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static const std::pair<GetCurrent, GetId> fns = [] {
    void* a = nullptr;
    void* b = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &q1) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess)
      a = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &q2) != cudaSuccess ||
        q2 != cudaDriverEntryPointSuccess)
      b = nullptr;
    return std::make_pair(reinterpret_cast<GetCurrent>(a), reinterpret_cast<GetId>(b));
  }();
  if (!fns.first || !fns.second) return false;
  CUcontext ctx = nullptr;
  if (fns.first(&ctx) != CUDA_SUCCESS || ctx == nullptr) return false;
  return fns.second(ctx, id) == CUDA_SUCCESS;
}

// The scratch array's device address on device `dev`, which the caller has made current. In host
// code the array's name is only a host-side stand-in, so the address is asked of the runtime
// (cudaGetSymbolAddress) with the device current: once per device and context, and again after
// the context was replaced. Without a context id it is looked up on every call.
int scratch_on(int dev, double** out) {
  unsigned long long id = 0;
  const bool have_id = current_context_id(&id);
  std::lock_guard<std::mutex> lk(g_mu);
  ScratchAddr& slot = g_addr[dev];
  if (!have_id || !slot.addr || slot.ctx_id != id) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_totals_scratch);
    if (e != cudaSuccess || p == nullptr) {
      slot = ScratchAddr{};
      return refuse(SHZ_E_CUDA, "cudaGetSymbolAddress of the totals scratch on device %d: %s", dev,
                    cudaGetErrorString(e));
    }
    slot.addr = static_cast<double*>(p);
    slot.ctx_id = have_id ? id : 0;
    if (!have_id) slot.addr = nullptr;  // nothing to check a cached address against: look up each call
    *out = static_cast<double*>(p);
    return SHZ_OK;
  }
  *out = slot.addr;
  return SHZ_OK;
}

}  // namespace

extern "C" const char* shz_totals_noalloc_error(void) { return t_msg.c_str(); }

extern "C" int shz_totals_noalloc(const shz_config* cfg, const void* u1, const void* u2, double* out, void* stream) {
  if (!cfg || !u1 || !u2 || !out) return refuse(SHZ_E_CONFIG, "shz_totals_noalloc: null argument");
  for (int a = 0; a < 3; a++)
    if (cfg->n[a] < 1) return refuse(SHZ_E_CONFIG, "shz_totals_noalloc: n[%d] = %d", a, cfg->n[a]);
  const double cells = (double)cfg->n[0] * cfg->n[1] * cfg->n[2];
  const double max_cells = (double)SHZ_TOTALS_MAX_BLOCKS * SHZ_TOTALS_CELLS_PER_BLOCK;
  if (cells > max_cells)
    return refuse(SHZ_E_CONFIG,
                  "shz_totals_noalloc: %.0f cells exceed the static scratch's maximum of %.0f cells (%d rows of %d cells)",
                  cells, max_cells, SHZ_TOTALS_MAX_BLOCKS, SHZ_TOTALS_CELLS_PER_BLOCK);
  if (!(cfg->gamma > 1) || !(cfg->dx > 0) || !(cfg->rho_floor > 0) || !(cfg->p_floor > 0))
    return refuse(SHZ_E_CONFIG, "shz_totals_noalloc: gamma > 1, dx > 0 and positive floors are required");
  const int dev = cfg->device;
  if (dev < 0 || dev >= kMaxDevices)
    return refuse(SHZ_E_CONFIG, "shz_totals_noalloc: device index %d outside 0..%d", dev, kMaxDevices - 1);
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return refuse(SHZ_E_NODEV, "shz_totals_noalloc: no CUDA device");
  if (dev >= count) return refuse(SHZ_E_CONFIG, "shz_totals_noalloc: device %d, but %d device(s) present", dev, count);
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  // cudaSetDevice also makes the device's primary context current on this thread, which the
  // context check of the address lookup reads.
  if (cudaSetDevice(dev) != cudaSuccess) return refuse(SHZ_E_CUDA, "shz_totals_noalloc: cudaSetDevice(%d)", dev);

  double* scratch = nullptr;
  int rc = scratch_on(dev, &scratch);
  if (rc == SHZ_OK) {
    const int nd = shz::ndim_of_size(cfg->n);  // as a handle of this size has it
    shz::KParams P = {};
    P.dx = cfg->dx;
    for (int a = 0; a < 3; a++) P.n[a] = cfg->n[a];
    P.gamma = (float)cfg->gamma;
    P.gm1 = (float)(cfg->gamma - 1);
    P.rho_floor = (float)cfg->rho_floor;
    P.p_floor = (float)cfg->p_floor;
    P.dv = std::pow(cfg->dx, nd);
    const size_t ncell = (size_t)cells;
    const int blocks = (int)((ncell + SHZ_TOTALS_CELLS_PER_BLOCK - 1) / SHZ_TOTALS_CELLS_PER_BLOCK);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Every row 0..blocks-1 is written by its block before the final kernel reads it, so
    // nothing left in the array by an earlier call is read and nothing needs clearing first.
    shz::diag_partial_kernel<<<blocks, 256, 0, s>>>(P, static_cast<const float4*>(u1), static_cast<const float4*>(u2),
                                                    ncell, scratch);
    shz::diag_final_kernel<<<1, 32, 0, s>>>(scratch, blocks, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = refuse(SHZ_E_CUDA, "shz_totals_noalloc: launch: %s", cudaGetErrorString(e));
  }
  if (prev >= 0 && prev != dev) cudaSetDevice(prev);
  return rc;
}
