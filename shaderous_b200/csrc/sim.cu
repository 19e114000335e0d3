// The C ABI of include/shaderous_b200.h: one simulation handle per uniform grid.
//
// The handle stands where the reference's Sim (src/sim.ts:1938) stands behind its Simulation
// interface (src/sim.ts:465-628): it owns the device state (two float4 arrays per parity, as
// the reference's 2x2 rgba32f textures, src/sim.ts:2301), the device clock and one stream, and
// enqueues a step as clock_kernel + sweep_kernel (sweep.cu). run() follows src/ui/api.ts:538:
// batches of steps whose clock is read back between batches; dt never leaves the device.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/shaderous_b200.h"
#include "problems.h"
#include "sweep.h"
#include "tune.h"

struct shz_sim {
  shz_config cfg;
  int ndim = 1;
  size_t ncell = 0;
  shz::KParams kp;
  float4* u1[2] = {nullptr, nullptr};  // first interior plane of each parity
  float4* u2[2] = {nullptr, nullptr};
  float4* a1[2] = {nullptr, nullptr};  // the allocations: halo planes below, the grid, halo planes above
  float4* a2[2] = {nullptr, nullptr};
  int halo_lo = 0, halo_hi = 0;        // stored ghost planes below and above (z faces of code 3)
  shz::SweepMaps maps[2];              // 3D: tensor maps of each parity for the sweep's TMA staging
  int* d_err = nullptr;                // the kernels' error word (a bounded wait that ran out)
  int cur = 0;
  shz::DevClock* clk = nullptr;
  unsigned* rates = nullptr;  // two slots
  int slot = 0;               // slot the next clock kernel reads
  double* diag_part = nullptr;
  double* diag_out = nullptr;
  cudaStream_t stream = nullptr;
  int device = 0;
  long long launches = 0;
  std::string err;
};

namespace {

std::mutex g_err_mu;
std::string g_err;

int fail(shz_sim* s, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (s) {
    s->err = buf;
  } else {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err = buf;
  }
  return code;
}

#define CUDA_OR_FAIL(sim, call)                                                                        \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess)                                                                              \
      return fail(sim, e_ == cudaErrorMemoryAllocation ? SHZ_E_OOM : SHZ_E_CUDA, "%s: %s", #call,       \
                  cudaGetErrorString(e_));                                                              \
  } while (0)

// Selects the handle's device for the duration of an ABI call (the library has its own CUDA
// runtime state, so the caller's current device is not assumed).
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int ndim_of(const shz_config& c) { return shz::ndim_of_size(c.n); }
// Ghost planes a halo face stores: the z march reads 1 + 2 planes beyond the slab with PPM's
// five-cell stencil, 1 + 1 with the three-cell limiters.
int halo_planes(const shz_config& c) { return c.recon == SHZ_RECON_PPM ? 3 : 2; }

int validate(const shz_config& c, std::string& why) {
  char b[256];
  for (int a = 0; a < 3; a++) {
    if (c.n[a] < 1) { snprintf(b, sizeof b, "n[%d] = %d: every axis needs at least one cell", a, c.n[a]); why = b; return -1; }
    const int top = a == 2 ? 3 : 2;
    if (c.bc_lo[a] < 0 || c.bc_lo[a] > top || c.bc_hi[a] < 0 || c.bc_hi[a] > top) {
      snprintf(b, sizeof b, "axis %d: boundary codes are 0 periodic, 1 outflow, 2 reflect (and 3 halo on z)", a);
      why = b;
      return -1;
    }
  }
  if (c.n[1] == 1 && c.n[2] > 1) { why = "a collapsed y axis with z cells: collapse z first (2D grids are x-y)"; return -1; }
  const int nd = ndim_of(c);
  if ((c.bc_lo[2] == 3 || c.bc_hi[2] == 3) && nd != 3) { why = "halo faces (code 3) are z faces of a 3D slab"; return -1; }
  if ((c.bc_lo[2] == 3) != (c.bc_hi[2] == 3) && (c.bc_lo[2] == 0 || c.bc_hi[2] == 0)) {
    why = "a periodic z face needs a periodic partner: use halo faces on both sides of a slab of a periodic grid";
    return -1;
  }
  const int need = shz::sweep_min_cells(c.recon);
  for (int a = 0; a < nd; a++)
    if (c.n[a] < need) { snprintf(b, sizeof b, "axis %d has %d cells; this reconstruction needs %d", a, c.n[a], need); why = b; return -1; }
  for (int a = nd; a < 3; a++)
    if (c.bc_lo[a] == 2 || c.bc_hi[a] == 2) {
      snprintf(b, sizeof b, "collapsed axis %d cannot reflect: use periodic or outflow", a); why = b; return -1;
    }
  if (!(c.dx > 0) || !std::isfinite(c.dx)) { why = "dx must be positive"; return -1; }
  if (!(c.gamma > 1)) { why = "gamma must exceed 1 (ideal gas)"; return -1; }
  if (!(c.cfl > 0)) { why = "cfl must be positive"; return -1; }
  if (!(c.rho_floor > 0) || !(c.p_floor > 0)) { why = "floors must be positive"; return -1; }
  if (c.riemann != SHZ_RIEMANN_HLLC && c.riemann != SHZ_RIEMANN_HLL) { why = "riemann must be HLLC (0) or HLL (1)"; return -1; }
  if (c.recon < SHZ_RECON_MINMOD || c.recon > SHZ_RECON_PPM) { why = "recon must be 0..4"; return -1; }
  if (c.signal_dims < 1 || c.signal_dims > 3) { why = "signal_dims must be 1, 2 or 3"; return -1; }
  if ((double)c.n[0] * c.n[1] * c.n[2] > 4.0e9) { why = "more than 4e9 cells"; return -1; }
  return 0;
}

void fill_kparams(shz_sim* s) {
  const shz_config& c = s->cfg;
  shz::KParams& k = s->kp;
  k.dx = c.dx;
  for (int a = 0; a < 3; a++) { k.n[a] = c.n[a]; k.bc_lo[a] = c.bc_lo[a]; k.bc_hi[a] = c.bc_hi[a]; }
  k.gamma = (float)c.gamma;
  k.gm1 = (float)(c.gamma - 1);
  k.inv_gm1 = (float)(1.0 / (c.gamma - 1));
  k.inv_gamma = (float)(1.0 / c.gamma);
  k.rho_floor = (float)c.rho_floor;
  k.p_floor = (float)c.p_floor;
  k.e_floor = (float)(c.p_floor / (c.gamma - 1));
  k.eta_dual = (float)c.eta_dual;
  k.shock_thresh = (float)c.shock_thresh;
  k.signal = (float)c.signal_dims;
  k.hll = c.riemann == SHZ_RIEMANN_HLL ? 1 : 0;
  k.dv = std::pow(c.dx, s->ndim);
}

int write_clock(shz_sim* s, double t, long long steps) {
  shz::DevClock h;
  std::memset(&h, 0, sizeof h);
  h.t = t;
  h.dt = 0;
  h.t_end = s->cfg.t_end;
  h.dt_max = s->cfg.dt_max;
  h.cfl_dx = s->cfg.cfl * s->cfg.dx;
  h.last_dt = 0;
  h.steps = steps;
  h.max_steps = std::numeric_limits<long long>::max();
  h.held = 0;
  h.bad = 0;
  CUDA_OR_FAIL(s, cudaMemcpyAsync(s->clk, &h, sizeof h, cudaMemcpyHostToDevice, s->stream));
  CUDA_OR_FAIL(s, cudaStreamSynchronize(s->stream));
  return 0;
}

// The kernels' error word: a bounded wait inside the sweep that ran out fails the call.
int check_err(shz_sim* s) {
  int e = 0;
  CUDA_OR_FAIL(s, cudaMemcpyAsync(&e, s->d_err, sizeof e, cudaMemcpyDeviceToHost, s->stream));
  CUDA_OR_FAIL(s, cudaStreamSynchronize(s->stream));
  if (e) {
    cudaMemsetAsync(s->d_err, 0, sizeof(int), s->stream);
    return fail(s, SHZ_E_TIMEOUT, "the sweep's bounded wait for a bulk copy ran out (code %d); the state is not valid", e);
  }
  return 0;
}

int read_clock(shz_sim* s, shz::DevClock* h) {
  CUDA_OR_FAIL(s, cudaMemcpyAsync(h, s->clk, sizeof *h, cudaMemcpyDeviceToHost, s->stream));
  CUDA_OR_FAIL(s, cudaStreamSynchronize(s->stream));
  return check_err(s);
}

// The rate maximum of the current state into the slot the next clock kernel reads.
int refresh_rate(shz_sim* s) {
  CUDA_OR_FAIL(s, shz::launch_rate(s->kp, s->u1[s->cur], s->u2[s->cur], s->ncell, s->rates + s->slot, s->stream));
  s->launches += 2;
  return 0;
}

// The autotuner's key of this grid's sweep, and its depth: in 3D the planes a CTA marches along z
// (0: the default); in 2D the rows a CTA marches along y, 0 for the tile form. Which 2D form runs
// is fixed by the grid's size, not by timing: the two forms are different kernels, which agree to
// rounding (the compiler may contract a multiply and an add differently in each), while every
// depth of one form is the same kernel and gives the same bits. 2D grids of at least 512 cells a
// side march along y, at a tuned depth (16 rows untuned); smaller ones take the tile form.
shz::tune::Key sweep_key(const shz_sim* s) {
  return shz::tune::Key{shz::tune::K_UNIFORM_SWEEP, s->ndim, s->cfg.recon,
                        (s->cfg.isentropic != 0 && s->cfg.recon != SHZ_RECON_PPM) ? 1 : 0,
                        shz::tune::size_class((long long)s->ncell)};
}
constexpr int ROWS_MIN_SIDE = 512, ROWS_DEFAULT = 16;
bool rows_form(const shz_sim* s) { return s->ndim == 2 && s->cfg.n[0] >= ROWS_MIN_SIDE && s->cfg.n[1] >= ROWS_MIN_SIDE; }
int sweep_tz(const shz_sim* s) {
  shz::tune::Choice c;
  if (s->ndim >= 2 && shz::tune::pinned(shz::tune::K_UNIFORM_SWEEP, &c)) return c.tz;
  if (s->ndim == 3) return shz::tune::lookup(sweep_key(s), &c) ? c.tz : 0;
  if (!rows_form(s)) return 0;
  return shz::tune::lookup(sweep_key(s), &c) ? c.tz : ROWS_DEFAULT;
}
bool wants_tuning(const shz_sim* s) {
  shz::tune::Choice c;
  return (s->ndim == 3 || rows_form(s)) && !shz::tune::pinned(shz::tune::K_UNIFORM_SWEEP, &c) &&
         shz::tune::needs(sweep_key(s));
}

// One step whose sweep is run once per candidate depth (z planes in 3D, y rows in 2D), timed, the
// fastest kept. The sweep reads one parity and writes the other (and folds the
// same rate maximum), so the step's result is that of a single launch. A clock held at its stop time is not tuned on (the sweep would
// only copy the state).
int tuned_step(shz_sim* s) {
  CUDA_OR_FAIL(s, shz::launch_clock(s->clk, s->rates, s->slot, s->stream));
  s->launches += 1;
  shz::DevClock h;
  CUDA_OR_FAIL(s, cudaMemcpyAsync(&h, s->clk, sizeof h, cudaMemcpyDeviceToHost, s->stream));
  CUDA_OR_FAIL(s, cudaStreamSynchronize(s->stream));
  auto launch = [&](const shz::tune::Choice& c) {
    return shz::launch_sweep(s->kp, s->ndim, s->cfg.recon, s->cfg.isentropic != 0, s->u1[s->cur], s->u2[s->cur],
                             s->u1[1 - s->cur], s->u2[1 - s->cur], s->clk, s->rates + (s->slot ^ 1), s->stream, c.tz, &s->maps[s->cur], s->d_err);
  };
  if (h.held) {
    CUDA_OR_FAIL(s, launch(shz::tune::Choice{}));
    s->launches += 1;
  } else {
    std::vector<shz::tune::Choice> cands;
    if (s->ndim == 3) {
      for (int tz : {shz::SWEEP_TZ_DEFAULT, 32, 128, 256}) {
        if (tz != shz::SWEEP_TZ_DEFAULT && tz > s->cfg.n[2]) continue;
        shz::tune::Choice c;
        c.tz = tz;
        cands.push_back(c);
      }
    } else {
      // the march along y at 8-64 rows a CTA (deeper marches leave too few CTAs)
      for (int rows : {ROWS_DEFAULT, 8, 32, 64}) {
        shz::tune::Choice c;
        c.tz = rows;
        cands.push_back(c);
      }
    }
    const int reps = 2;
    shz::tune::Choice best;
    CUDA_OR_FAIL(s, shz::tune::choose(sweep_key(s), cands, launch, s->stream, reps, &best));
    s->launches += (long long)cands.size() * (1 + reps);
  }
  s->cur ^= 1;
  s->slot ^= 1;
  return 0;
}

int enqueue_steps(shz_sim* s, int n) {
  for (int i = 0; i < n; i++) {
    if (wants_tuning(s)) {
      const int rc = tuned_step(s);
      if (rc) return rc;
      continue;
    }
    CUDA_OR_FAIL(s, shz::launch_clock(s->clk, s->rates, s->slot, s->stream));
    CUDA_OR_FAIL(s, shz::launch_sweep(s->kp, s->ndim, s->cfg.recon, s->cfg.isentropic != 0, s->u1[s->cur], s->u2[s->cur],
                                      s->u1[1 - s->cur], s->u2[1 - s->cur], s->clk, s->rates + (s->slot ^ 1), s->stream,
                                      sweep_tz(s), &s->maps[s->cur], s->d_err));
    s->launches += 2;
    s->cur ^= 1;
    s->slot ^= 1;
  }
  return 0;
}

}  // namespace

extern "C" {

const char* shz_version(void) { return "shaderous_b200 0.1.0 (sm_100a)"; }

int shz_config_default(shz_config* c, int32_t nx, int32_t ny, int32_t nz, double dx) {
  if (!c) return SHZ_E_CONFIG;
  std::memset(c, 0, sizeof *c);
  c->n[0] = nx; c->n[1] = ny; c->n[2] = nz;
  c->dx = dx;
  c->gamma = 5.0 / 3.0;
  for (int a = 0; a < 3; a++) { c->bc_lo[a] = SHZ_BC_PERIODIC; c->bc_hi[a] = SHZ_BC_PERIODIC; }
  // configFor defaults (src/sim.ts:672-705)
  c->cfl = 0.8;
  c->rho_floor = 1e-10;
  c->p_floor = 1e-14;
  c->eta_dual = 1e-3;
  c->shock_thresh = 0.5;
  c->riemann = SHZ_RIEMANN_HLLC;
  c->recon = SHZ_RECON_KOREN;
  c->isentropic = 1;
  c->signal_dims = 3;
  c->t_end = HUGE_VAL;
  c->dt_max = HUGE_VAL;
  return 0;
}

const char* shz_last_error(const shz_sim* sim) {
  if (sim) return sim->err.c_str();
  std::lock_guard<std::mutex> lk(g_err_mu);
  return g_err.c_str();
}

int shz_create(const shz_config* cfg, shz_sim** out) {
  if (!cfg || !out) return fail(nullptr, SHZ_E_CONFIG, "shz_create: null argument");
  *out = nullptr;
  std::string why;
  if (validate(*cfg, why) != 0) return fail(nullptr, SHZ_E_CONFIG, "refused configuration: %s", why.c_str());
  const int dev = cfg->device;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return fail(nullptr, SHZ_E_NODEV, "no CUDA device: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= count) return fail(nullptr, SHZ_E_CONFIG, "refused configuration: device %d of %d", dev, count);
  DeviceScope ds_(dev);
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, dev);
  if (e != cudaSuccess) return fail(nullptr, SHZ_E_NODEV, "cudaGetDeviceProperties: %s", cudaGetErrorString(e));
  if (prop.major != 10) return fail(nullptr, SHZ_E_NODEV, "device %s is sm_%d%d; this library is built for sm_100a", prop.name, prop.major, prop.minor);

  shz_sim* s = new shz_sim();
  s->cfg = *cfg;
  s->device = dev;
  s->ndim = ndim_of(*cfg);
  s->ncell = (size_t)cfg->n[0] * cfg->n[1] * cfg->n[2];
  fill_kparams(s);
  const size_t bytes = s->ncell * sizeof(float4);
  const size_t plane = (size_t)cfg->n[0] * cfg->n[1];
  const int hz = halo_planes(*cfg);
  s->halo_lo = cfg->bc_lo[2] == 3 ? hz : 0;
  s->halo_hi = cfg->bc_hi[2] == 3 ? hz : 0;
  const size_t abytes = bytes + (size_t)(s->halo_lo + s->halo_hi) * plane * sizeof(float4);
  auto bail = [&](int code) {
    std::string m = s->err;
    shz_destroy(s);
    return fail(nullptr, code, "%s", m.c_str());
  };
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { fail(s, SHZ_E_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e)); return bail(SHZ_E_CUDA); }
  for (int p = 0; p < 2; p++) {
    if (cudaMalloc(&s->a1[p], abytes) != cudaSuccess || cudaMalloc(&s->a2[p], abytes) != cudaSuccess) {
      cudaGetLastError();
      fail(s, SHZ_E_OOM, "device state of %zu cells (%.2f GB) does not fit", s->ncell, 4.0 * abytes / 1e9);
      return bail(SHZ_E_OOM);
    }
    s->u1[p] = s->a1[p] + (size_t)s->halo_lo * plane;
    s->u2[p] = s->a2[p] + (size_t)s->halo_lo * plane;
    if (s->ndim == 3)
      shz::encode_sweep_maps(&s->maps[p], s->a1[p], s->a2[p], cfg->n[0], cfg->n[1],
                             cfg->n[2] + s->halo_lo + s->halo_hi, s->halo_lo, cfg->recon);
    // (ghost planes start as zeros until the caller fills them: a state of zeros is a vacuum,
    // which the floors keep finite)
    cudaMemsetAsync(s->a1[p], 0, abytes, s->stream);
    cudaMemsetAsync(s->a2[p], 0, abytes, s->stream);
  }
  const int dblocks = shz::diag_blocks(s->ncell);
  if (cudaMalloc(&s->d_err, sizeof(int)) != cudaSuccess || cudaMemset(s->d_err, 0, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&s->clk, sizeof(shz::DevClock)) != cudaSuccess || cudaMalloc(&s->rates, 2 * sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&s->diag_part, (size_t)dblocks * 16 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&s->diag_out, 16 * sizeof(double)) != cudaSuccess) {  // the totals or the extended channels
    cudaGetLastError();
    fail(s, SHZ_E_OOM, "clock / reduction buffers do not fit");
    return bail(SHZ_E_OOM);
  }
  cudaMemsetAsync(s->rates, 0, 2 * sizeof(unsigned), s->stream);
  if (write_clock(s, 0.0, 0) != 0) return bail(SHZ_E_CUDA);
  *out = s;
  return SHZ_OK;
}

void shz_destroy(shz_sim* s) {
  if (!s) return;
  DeviceScope ds_(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (int p = 0; p < 2; p++) {
    if (s->a1[p]) cudaFree(s->a1[p]);
    if (s->a2[p]) cudaFree(s->a2[p]);
  }
  if (s->d_err) cudaFree(s->d_err);
  if (s->clk) cudaFree(s->clk);
  if (s->rates) cudaFree(s->rates);
  if (s->diag_part) cudaFree(s->diag_part);
  if (s->diag_out) cudaFree(s->diag_out);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

}  // extern "C"

namespace {
// The handle's planes as planes kofs.. of `prob` sampled on the grid `grid` (the handle's own
// grid with kofs 0, or the whole grid a slab belongs to); then the clock to 0 and the rate.
int reset_planes(shz_sim* s, const shz_config& grid, const shz_problem* prob, int kofs) {
  if (!shz::problem_known(prob->kind)) return fail(s, SHZ_E_CONFIG, "unknown problem kind %d", prob->kind);
  const int nx = s->cfg.n[0], ny = s->cfg.n[1], nz = s->cfg.n[2];
  const size_t plane = (size_t)nx * ny;
  // slabs of planes of at most ~32M cells, staged through pinned memory
  int kstep = (int)std::max<size_t>(1, (size_t)(32u << 20) / plane);
  if (kstep > nz) kstep = nz;
  std::vector<double> w((size_t)kstep * plane * 6);
  float* h1 = nullptr;
  float* h2 = nullptr;
  CUDA_OR_FAIL(s, cudaMallocHost(&h1, (size_t)kstep * plane * sizeof(float4)));
  if (cudaMallocHost(&h2, (size_t)kstep * plane * sizeof(float4)) != cudaSuccess) {
    cudaFreeHost(h1);
    return fail(s, SHZ_E_OOM, "pinned staging buffer");
  }
  int rc = 0;
  for (int k0 = 0; k0 < nz && rc == 0; k0 += kstep) {
    const int k1 = std::min(nz, k0 + kstep);
    const size_t cnt = (size_t)(k1 - k0) * plane;
    shz::problem_prims(grid, *prob, kofs + k0, kofs + k1, w.data());
    shz::prims_to_state(w.data(), s->cfg.gamma, (int64_t)cnt, h1, h2);
    cudaError_t e1 = cudaMemcpyAsync(s->u1[s->cur] + (size_t)k0 * plane, h1, cnt * sizeof(float4), cudaMemcpyHostToDevice, s->stream);
    cudaError_t e2 = cudaMemcpyAsync(s->u2[s->cur] + (size_t)k0 * plane, h2, cnt * sizeof(float4), cudaMemcpyHostToDevice, s->stream);
    cudaError_t e3 = cudaStreamSynchronize(s->stream);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
      rc = fail(s, SHZ_E_CUDA, "state upload: %s", cudaGetErrorString(e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3)));
  }
  cudaFreeHost(h1);
  cudaFreeHost(h2);
  if (rc) return rc;
  if ((rc = write_clock(s, 0.0, 0))) return rc;
  return refresh_rate(s);
}
}  // namespace

extern "C" {

int shz_reset_problem(shz_sim* s, const shz_problem* prob) {
  if (!s || !prob) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  return reset_planes(s, s->cfg, prob, 0);
}

int shz_reset_problem_slab(shz_sim* s, const shz_config* grid, const shz_problem* prob, int32_t k0) {
  if (!s || !grid || !prob) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  if (grid->n[0] != s->cfg.n[0] || grid->n[1] != s->cfg.n[1] || grid->dx != s->cfg.dx)
    return fail(s, SHZ_E_CONFIG, "the whole grid must have the slab's nx, ny and dx");
  if (k0 < 0 || (int64_t)k0 + s->cfg.n[2] > grid->n[2])
    return fail(s, SHZ_E_CONFIG, "planes %d..%d are not planes of the whole grid (nz %d)", k0, k0 + s->cfg.n[2] - 1,
                grid->n[2]);
  return reset_planes(s, *grid, prob, k0);
}

int shz_set_state(shz_sim* s, const float* u1, const float* u2, size_t ncell) {
  if (!s || !u1 || !u2) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  if (ncell != s->ncell) return fail(s, SHZ_E_CONFIG, "set_state: %zu cells given, the grid has %zu", ncell, s->ncell);
  CUDA_OR_FAIL(s, cudaMemcpyAsync(s->u1[s->cur], u1, ncell * sizeof(float4), cudaMemcpyHostToDevice, s->stream));
  CUDA_OR_FAIL(s, cudaMemcpyAsync(s->u2[s->cur], u2, ncell * sizeof(float4), cudaMemcpyHostToDevice, s->stream));
  return refresh_rate(s);
}

int shz_get_state(shz_sim* s, float* u1, float* u2, size_t ncell) {
  if (!s || !u1 || !u2) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  if (ncell != s->ncell) return fail(s, SHZ_E_CONFIG, "get_state: room for %zu cells, the grid has %zu", ncell, s->ncell);
  CUDA_OR_FAIL(s, cudaMemcpyAsync(u1, s->u1[s->cur], ncell * sizeof(float4), cudaMemcpyDeviceToHost, s->stream));
  CUDA_OR_FAIL(s, cudaMemcpyAsync(u2, s->u2[s->cur], ncell * sizeof(float4), cudaMemcpyDeviceToHost, s->stream));
  CUDA_OR_FAIL(s, cudaStreamSynchronize(s->stream));
  return 0;
}

int shz_step(shz_sim* s, int32_t n) {
  if (!s) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  if (n < 0) return fail(s, SHZ_E_CONFIG, "step: n = %d", n);
  return enqueue_steps(s, n);
}

int shz_sync(shz_sim* s) {
  if (!s) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  CUDA_OR_FAIL(s, cudaStreamSynchronize(s->stream));
  return 0;
}

int shz_clock(shz_sim* s, double* t, double* dt, int64_t* steps) {
  if (!s) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  shz::DevClock h;
  int rc = read_clock(s, &h);
  if (rc) return rc;
  if (t) *t = h.t;
  if (dt) *dt = h.dt;
  if (steps) *steps = h.steps;
  if (h.bad) return fail(s, SHZ_E_NAN, "the clock is NaN after %lld steps", h.steps);
  return 0;
}

int shz_set_clock(shz_sim* s, double t, int64_t steps) {
  if (!s) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  return write_clock(s, t, steps);
}

int shz_set_t_end(shz_sim* s, double t_end) {
  if (!s) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  s->cfg.t_end = t_end;
  CUDA_OR_FAIL(s, cudaMemcpyAsync(&s->clk->t_end, &s->cfg.t_end, sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CUDA_OR_FAIL(s, cudaStreamSynchronize(s->stream));
  return 0;
}

int shz_run(shz_sim* s, const shz_run_opts* o, shz_run_result* r) {
  if (!s || !o || !r) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  const auto t0 = std::chrono::steady_clock::now();
  auto elapsed_ms = [&]() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  };
  const bool has_until = !std::isnan(o->until);
  if (o->steps < 0 && !has_until) return fail(s, SHZ_E_CONFIG, "run() needs `steps`, `until`, or both");
  shz::DevClock c;
  int rc = read_clock(s, &c);
  if (rc) return rc;
  const long long start = c.steps;
  double last_dt = c.last_dt;
  auto finish = [&](int stopped) {
    r->t = c.t;
    r->dt = c.dt;
    r->steps = c.steps;
    r->taken = c.steps - start;
    r->seconds = elapsed_ms() / 1000.0;
    r->stopped = stopped;
    r->last_dt = last_dt;
    return 0;
  };
  if (has_until && !(o->until > c.t)) return finish(SHZ_STOP_TIME);
  const double t_end_was = s->cfg.t_end;
  const double stop = has_until ? std::min(o->until, t_end_was) : t_end_was;
  if (stop != t_end_was) {
    CUDA_OR_FAIL(s, cudaMemcpyAsync(&s->clk->t_end, &stop, sizeof(double), cudaMemcpyHostToDevice, s->stream));
  }
  int stopped = -1;
  int grow = 1;
  double ms_per_step = 0;  // the batches' pace (api.ts run: batches of about BATCH_MS = 50 ms)
  for (;;) {
    const long long taken = c.steps - start;
    const long long left = o->steps < 0 ? std::numeric_limits<long long>::max() : o->steps - taken;
    if (left <= 0) { stopped = SHZ_STOP_STEPS; break; }
    if (has_until && c.t >= o->until * (1 - 1e-12)) { stopped = SHZ_STOP_TIME; break; }
    if (std::isfinite(t_end_was) && c.t >= t_end_was * (1 - 1e-12)) { stopped = SHZ_STOP_END; break; }
    if (o->timeout_ms > 0 && elapsed_ms() > o->timeout_ms) { stopped = SHZ_STOP_TIMEOUT; break; }
    long long batch = std::min<long long>(left, grow);
    if (ms_per_step > 0) batch = std::min<long long>(batch, std::max(1.0, std::floor(50.0 / ms_per_step)));
    if (std::isfinite(stop) && last_dt > 0) {
      const double ahead = std::ceil((stop - c.t) / last_dt - 1e-6);
      if (ahead >= 1 && ahead < (double)batch) batch = (long long)ahead;
    }
    if (batch < 1) batch = 1;
    const double b0 = elapsed_ms();
    if ((rc = enqueue_steps(s, (int)batch))) break;
    if ((rc = read_clock(s, &c))) break;
    if (c.bad) { rc = fail(s, SHZ_E_NAN, "the clock is NaN after %lld steps", c.steps); break; }
    if (c.last_dt > 0) last_dt = c.last_dt;
    if (c.steps - start == taken) {
      // nothing advanced: the clock is held at the stop
      stopped = has_until && c.t >= o->until * (1 - 1e-9) ? SHZ_STOP_TIME : SHZ_STOP_END;
      break;
    }
    const double m = (elapsed_ms() - b0) / (double)batch;
    ms_per_step = ms_per_step > 0 ? 0.7 * ms_per_step + 0.3 * m : m;
    grow = std::min(grow * 2, 256);
  }
  if (stop != t_end_was) {
    cudaMemcpyAsync(&s->clk->t_end, &t_end_was, sizeof(double), cudaMemcpyHostToDevice, s->stream);
    cudaStreamSynchronize(s->stream);
  }
  if (rc) return rc;
  return finish(stopped);
}

int shz_diagnostics(shz_sim* s, shz_diag* d) {
  if (!s || !d) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  CUDA_OR_FAIL(s, shz::launch_diag(s->kp, s->u1[s->cur], s->u2[s->cur], s->ncell, s->diag_part, s->diag_out, s->stream));
  s->launches += 2;
  double v[shz::DIAG_VALUES];
  CUDA_OR_FAIL(s, cudaMemcpyAsync(v, s->diag_out, sizeof v, cudaMemcpyDeviceToHost, s->stream));
  shz::DevClock c;
  int rc = read_clock(s, &c);
  if (rc) return rc;
  d->t = c.t;
  d->dt = c.dt;
  d->steps = c.steps;
  d->mass = v[0];
  d->momentum[0] = v[1];
  d->momentum[1] = v[2];
  d->momentum[2] = v[3];
  d->e_kin = v[4];
  d->e_int = v[5];
  d->e_tot = v[6];
  d->floored = v[7];
  d->max_mach = v[8];
  return 0;
}

int shz_diagnostics_ext(shz_sim* s, shz_diag_ext* d) {
  if (!s || !d) return SHZ_E_CONFIG;
  int rc = shz_diagnostics(s, &d->base);
  if (rc) return rc;
  DeviceScope ds_(s->device);
  CUDA_OR_FAIL(s, shz::launch_diag_ext(s->kp, s->u1[s->cur], s->u2[s->cur], s->ncell, s->diag_part, s->diag_out,
                                       s->stream));
  s->launches += 2;
  double v[shz::DIAG_EXT_VALUES];
  CUDA_OR_FAIL(s, cudaMemcpyAsync(v, s->diag_out, sizeof v, cudaMemcpyDeviceToHost, s->stream));
  CUDA_OR_FAIL(s, cudaStreamSynchronize(s->stream));
  for (int i = 0; i < 5; i++) {
    d->range[i][0] = v[i];
    d->range[i][1] = v[5 + i];
  }
  for (int i = 0; i < 3; i++) d->com[i] = d->base.mass > 0 ? v[10 + i] / d->base.mass : 0.0;
  d->e_grav = 0.0;
  d->jeans_unresolved = 0.0;
  d->nuclear_heating = 0.0;
  return 0;
}

int shz_state_device(shz_sim* s, void** u1, void** u2) {
  if (!s || !u1 || !u2) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  *u1 = s->u1[s->cur];
  *u2 = s->u2[s->cur];
  return 0;
}

int shz_halo_depth(const shz_sim* s, int32_t* planes) {
  if (!s || !planes) return SHZ_E_CONFIG;
  *planes = halo_planes(s->cfg);
  return 0;
}

int shz_halo_device(shz_sim* s, int32_t side, void** inner_u1, void** inner_u2, void** ghost_u1, void** ghost_u2,
                    size_t* bytes) {
  if (!s || (side != 0 && side != 1) || !inner_u1 || !inner_u2 || !ghost_u1 || !ghost_u2 || !bytes) return SHZ_E_CONFIG;
  const int depth = side == 0 ? s->halo_lo : s->halo_hi;
  if (depth == 0) return fail(s, SHZ_E_CONFIG, "z face %d is not a halo face (code 3)", side);
  const size_t plane = (size_t)s->cfg.n[0] * s->cfg.n[1];
  const size_t nz = (size_t)s->cfg.n[2];
  if (nz < (size_t)depth) return fail(s, SHZ_E_CONFIG, "the slab has fewer planes than its halo");
  // inner: the `depth` planes next to the face; ghost: the `depth` stored planes beyond it
  const size_t in0 = side == 0 ? 0 : (nz - depth) * plane;
  const ptrdiff_t g0 = side == 0 ? -(ptrdiff_t)(depth * plane) : (ptrdiff_t)(nz * plane);
  *inner_u1 = s->u1[s->cur] + in0;
  *inner_u2 = s->u2[s->cur] + in0;
  *ghost_u1 = s->u1[s->cur] + g0;
  *ghost_u2 = s->u2[s->cur] + g0;
  *bytes = (size_t)depth * plane * sizeof(float4);
  return 0;
}

int shz_rate_device(shz_sim* s, void** rate) {
  if (!s || !rate) return SHZ_E_CONFIG;
  *rate = s->rates + s->slot;
  return 0;
}

int shz_stream(shz_sim* s, void** stream) {
  if (!s || !stream) return SHZ_E_CONFIG;
  *stream = (void*)s->stream;
  return 0;
}

int shz_profile(shz_sim* s, int32_t n, shz_profile_result* out) {
  if (!s || !out || n < 1) return SHZ_E_CONFIG;
  DeviceScope ds_(s->device);
  std::vector<cudaEvent_t> ev(2 * (size_t)n + 1);
  for (auto& e : ev) CUDA_OR_FAIL(s, cudaEventCreate(&e));
  const long long l0 = s->launches;
  int rc = 0;
  CUDA_OR_FAIL(s, cudaEventRecord(ev[0], s->stream));
  for (int i = 0; i < n && rc == 0; i++) {
    if (wants_tuning(s)) {
      // (a step that tunes the sweep counts whole, tuning included, as sweep time)
      CUDA_OR_FAIL(s, cudaEventRecord(ev[1 + 2 * i], s->stream));
      rc = tuned_step(s);
      if (rc == 0) CUDA_OR_FAIL(s, cudaEventRecord(ev[2 + 2 * i], s->stream));
      continue;
    }
    cudaError_t e = shz::launch_clock(s->clk, s->rates, s->slot, s->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev[1 + 2 * i], s->stream);
    if (e == cudaSuccess)
      e = shz::launch_sweep(s->kp, s->ndim, s->cfg.recon, s->cfg.isentropic != 0, s->u1[s->cur], s->u2[s->cur],
                            s->u1[1 - s->cur], s->u2[1 - s->cur], s->clk, s->rates + (s->slot ^ 1), s->stream,
                            sweep_tz(s), &s->maps[s->cur], s->d_err);
    if (e == cudaSuccess) e = cudaEventRecord(ev[2 + 2 * i], s->stream);
    if (e != cudaSuccess) rc = fail(s, SHZ_E_CUDA, "profile step %d: %s", i, cudaGetErrorString(e));
    s->launches += 2;
    s->cur ^= 1;
    s->slot ^= 1;
  }
  if (rc == 0) {
    cudaError_t e = cudaEventSynchronize(ev[2 * (size_t)n]);
    if (e != cudaSuccess) rc = fail(s, SHZ_E_CUDA, "profile sync: %s", cudaGetErrorString(e));
    if (rc == 0) rc = check_err(s);
  }
  if (rc == 0) {
    float tot = 0.f;
    double sw = 0.0;
    cudaEventElapsedTime(&tot, ev[0], ev[2 * (size_t)n]);
    for (int i = 0; i < n; i++) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[1 + 2 * i], ev[2 + 2 * i]);
      sw += ms;
    }
    out->steps = n;
    out->total_ms = tot;
    out->sweep_ms = sw;
    out->launches = s->launches - l0;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return rc;
}

int64_t shz_kernel_launches(const shz_sim* s) { return s ? s->launches : 0; }

}  // extern "C"
