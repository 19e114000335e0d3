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
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/shaderous_b200.h"
#include "hydro_math.cuh"

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
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};  // device address of g_totals_scratch, per device, once set up
std::string g_msg;

int refuse(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  std::lock_guard<std::mutex> lk(g_mu);
  g_msg = buf;
  return code;
}

// The scratch array's device address on the current device. In host code the array's name is
// only a host-side stand-in, so the address is asked of the runtime once per device, with that
// device current.
int scratch_on(int dev, double** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_totals_scratch);
    if (e != cudaSuccess || p == nullptr) {
      char buf[256];
      snprintf(buf, sizeof buf, "cudaGetSymbolAddress of the totals scratch on device %d: %s", dev,
               cudaGetErrorString(e));
      g_msg = buf;
      return SHZ_E_CUDA;
    }
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return SHZ_OK;
}

}  // namespace

extern "C" const char* shz_totals_noalloc_error(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  return g_msg.c_str();
}

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
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return refuse(SHZ_E_NODEV, "shz_totals_noalloc: no CUDA device");
  const int dev = cfg->device;
  if (dev < 0 || dev >= count || dev >= kMaxDevices) return refuse(SHZ_E_CONFIG, "shz_totals_noalloc: device %d of %d", dev, count);
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (prev != dev && cudaSetDevice(dev) != cudaSuccess) return refuse(SHZ_E_CUDA, "shz_totals_noalloc: cudaSetDevice(%d)", dev);

  double* scratch = nullptr;
  int rc = scratch_on(dev, &scratch);
  if (rc == SHZ_OK) {
    const int nd = cfg->n[2] > 1 ? 3 : (cfg->n[1] > 1 ? 2 : 1);
    shz::KParams P = {};
    P.dx = cfg->dx;
    for (int a = 0; a < 3; a++) P.n[a] = cfg->n[a];
    P.gamma = (float)cfg->gamma;
    P.gm1 = (float)(cfg->gamma - 1);
    P.rho_floor = (float)cfg->rho_floor;
    P.p_floor = (float)cfg->p_floor;
    P.dv = (float)std::pow(cfg->dx, nd);
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
