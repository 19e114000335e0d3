// Serving: many independent hydro requests resident in HBM, advanced together by the adaptive
// grid's block passes (amr_kernels.cu) over one work list, with continuous batching.
//
// Each request is a uniform grid of 16^ndim-cell blocks: a level-0 block tree whose rows the
// server writes into one shared block table, with the request's own parameter and clock index in
// word 26. An engine per dimensionality owns the shared atlases; a round is `round_steps` steps,
// each one CUDA graph of three kernels (assemble, clocks, the fused block sweep) over the blocks of
// every running request. Between rounds the
// host reads the clocks back, finishes the requests that have taken their steps (float64 totals,
// optionally their state), frees their slots, and admits queued requests whose blocks fit, their
// initial states sampled on the host while the GPU runs the round.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <limits>
#include <memory>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/shaderous_b200.h"
#include "amr_kernels.h"
#include "amr_tree.h"
#include "problems.h"
#include "sweep.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr int BS = 16;

struct Grid {
  int64_t id = 0;
  shz_request req;
  int eng = 0;  // 0: 2D, 1: 3D
  int g = -1;   // parameter and clock index in the engine
  int nblocks = 0;
  std::vector<int> slots;             // global slot per local block (local = root-block order)
  std::vector<int32_t> rows;          // the request's block-table rows with local neighbour slots
  std::vector<float4> s1, s2;         // staged initial state, local block order
  bool staged = false;
  double arrival = 0, finished = 0;
  bool done = false;
  bool cancelled = false;  // shz_server_cancel took it off the queue or the device
  // A large request run as a uniform grid (direct_large): its handle, the steps enqueued so far,
  // its device bytes, and its span's events for the busy time.
  bool direct = false;
  shz_sim* sim = nullptr;
  int enq = 0;
  double bytes = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  shz_diag diag{};
  std::vector<float> out1, out2;      // final state (keep_states), uniform layout
};

struct Engine {
  int ndim = 3, CB = 0, WN = 0;
  int cap = 0, gmax = 0;
  float4* u1[2] = {nullptr, nullptr};
  float4* u2[2] = {nullptr, nullptr};
  float4 *w1 = nullptr, *w2 = nullptr;
  int *d_bt = nullptr, *d_list = nullptr, *d_glist = nullptr;
  int* d_rest = nullptr;  // the split assemble's second-pass blocks (none on uniform grids' blocks)
  std::vector<int32_t> h_rest;
  shz::KParams* d_gp = nullptr;
  shz::DevClock* d_clk = nullptr;
  unsigned* d_rates = nullptr;
  double *d_part = nullptr, *d_out = nullptr;
  int* d_err = nullptr;  // the kernels' error word
  std::vector<int> free_slots, free_g;
  std::vector<Grid*> active;
  std::vector<int32_t> h_bt, h_list;
  shz::DevClock* h_clk = nullptr;  // pinned, so that the per-round readback stays asynchronous
  int high = 0;  // rows of the table in use: slots below this may be live
  int cur = 0, rslot = 0;
  bool dirty = true;
  cudaGraphExec_t graphs[4] = {nullptr, nullptr, nullptr, nullptr};
  long long graph_launches[4] = {0, 0, 0, 0};  // kernels one replay of each graph launches
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // a round's span on this engine's stream
  shz::AmrLaunch L{};
  long long launches = 0;
  int64_t slot_bytes() const { return (int64_t)(4 * CB + 2 * WN) * 16; }
};

}  // namespace

struct shz_server {
  shz_server_config cfg;
  Engine e[2];
  std::deque<Grid*> pending;
  std::unordered_map<int64_t, std::unique_ptr<Grid>> grids;
  int64_t next_id = 1;
  std::string err;
  int device = 0;
  Clock::time_point t0 = Clock::now();
  long long rounds = 0;
  long long max_concurrent = 0;
  double busy_s = 0;  // GPU seconds of the rounds: per round the longest stream's event span
  // large requests run as uniform grids (direct_large): the running ones, their device bytes
  // against their share of the budget, and the kernels their handles launched
  std::vector<Grid*> direct;
  double direct_budget = 0, direct_used = 0;
  long long direct_launches = 0;
};

namespace {

int fail(shz_server* s, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (s) s->err = buf;
  return code;
}
std::string g_create_err;

#define SV_CUDA(s, call)                                                                                 \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess)                                                                               \
      return fail(s, e_ == cudaErrorMemoryAllocation ? SHZ_E_OOM : SHZ_E_CUDA, "%s: %s", #call,         \
                  cudaGetErrorString(e_));                                                               \
  } while (0)

struct Dev {
  int prev = -1;
  explicit Dev(int d) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != d) cudaSetDevice(d);
  }
  ~Dev() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

double now_s(const shz_server* s) { return std::chrono::duration<double>(Clock::now() - s->t0).count(); }

// Requests this large run as uniform grids when the server has direct_large: the fused sweep of a
// whole grid fills the GPU at these sizes, where the block passes' ghost-filled atlases cost more.
constexpr int DIRECT_MAX = 8;  // uniform grids running at once
bool direct_size(const shz_request& r) {
  const double cells = std::pow((double)r.n, r.ndim);
  return cells >= (r.ndim == 3 ? (double)(1 << 21) : (double)(1 << 18));
}
// Device bytes of a request run as a uniform grid: two parities of (u1, u2), and the handle's rest.
double direct_bytes(const shz_request& r) { return std::pow((double)r.n, r.ndim) * 64.0 + (16 << 20); }

bool running(const shz_server* s) { return !s->e[0].active.empty() || !s->e[1].active.empty() || !s->direct.empty(); }

void drop_graphs(Engine& e) {
  for (auto& g : e.graphs)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

int engine_init(shz_server* s, Engine& e, int ndim, double budget) {
  e.ndim = ndim;
  e.CB = ndim == 3 ? 4096 : 256;
  e.WN = ndim == 3 ? 8000 : 400;
  e.gmax = s->cfg.max_grids;
  e.cap = (int)std::max<int64_t>(0, (int64_t)(budget / (double)e.slot_bytes()));
  e.L.ndim = ndim;
  e.L.recon = s->cfg.hydro.recon;
  e.L.isen = s->cfg.hydro.isentropic != 0;
  if (e.cap == 0) return 0;
  SV_CUDA(s, cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking));
  const size_t cap = e.cap;
  for (int p = 0; p < 2; p++) {
    SV_CUDA(s, cudaMalloc(&e.u1[p], cap * e.CB * sizeof(float4)));
    SV_CUDA(s, cudaMalloc(&e.u2[p], cap * e.CB * sizeof(float4)));
  }
  SV_CUDA(s, cudaMalloc(&e.w1, cap * e.WN * sizeof(float4)));
  SV_CUDA(s, cudaMalloc(&e.w2, cap * e.WN * sizeof(float4)));
  SV_CUDA(s, cudaMalloc(&e.d_err, sizeof(int)));
  SV_CUDA(s, cudaMemset(e.d_err, 0, sizeof(int)));
  SV_CUDA(s, cudaMalloc(&e.d_bt, cap * 32 * sizeof(int)));
  SV_CUDA(s, cudaMalloc(&e.d_list, cap * sizeof(int)));
  SV_CUDA(s, cudaMalloc(&e.d_glist, cap * sizeof(int)));
  SV_CUDA(s, cudaMalloc(&e.d_rest, cap * sizeof(int)));
  SV_CUDA(s, cudaMalloc(&e.d_gp, e.gmax * sizeof(shz::KParams)));
  SV_CUDA(s, cudaMalloc(&e.d_clk, e.gmax * sizeof(shz::DevClock)));
  SV_CUDA(s, cudaMalloc(&e.d_rates, 2 * e.gmax * sizeof(unsigned)));
  SV_CUDA(s, cudaMalloc(&e.d_part, (size_t)shz::amr_diag_blocks(e.cap) * 9 * sizeof(double)));
  SV_CUDA(s, cudaMalloc(&e.d_out, 9 * sizeof(double)));
  SV_CUDA(s, cudaMemset(e.d_rates, 0, 2 * e.gmax * sizeof(unsigned)));
  // idle clocks hold (max_steps 0) so that unused indices never step
  std::vector<shz::DevClock> idle(e.gmax);
  for (auto& c : idle) {
    std::memset(&c, 0, sizeof c);
    c.t_end = HUGE_VAL;
    c.dt_max = HUGE_VAL;
    c.cfl_dx = 1.0;
  }
  SV_CUDA(s, cudaMemcpy(e.d_clk, idle.data(), e.gmax * sizeof(shz::DevClock), cudaMemcpyHostToDevice));
  SV_CUDA(s, cudaMallocHost(&e.h_clk, e.gmax * sizeof(shz::DevClock)));
  e.h_bt.assign(cap * 32, -1);
  for (int i = e.cap - 1; i >= 0; i--) e.free_slots.push_back(i);
  for (int i = e.gmax - 1; i >= 0; i--) e.free_g.push_back(i);
  e.L.gp = e.d_gp;
  e.L.bt = e.d_bt;
  e.L.w1 = e.w1;
  e.L.w2 = e.w2;
  e.L.err = e.d_err;
  e.L.p1 = nullptr;  // (the fused sweep keeps no half-step atlas)
  e.L.p2 = nullptr;
  return 0;
}

void engine_free(Engine& e) {
  drop_graphs(e);
  if (e.stream) cudaStreamSynchronize(e.stream);
  for (int p = 0; p < 2; p++) {
    cudaFree(e.u1[p]);
    cudaFree(e.u2[p]);
  }
  void* b[] = {e.w1, e.w2, e.d_err, e.d_bt, e.d_list, e.d_glist, e.d_gp, e.d_clk, e.d_rates, e.d_part, e.d_out, e.d_rest};
  for (void* x : b)
    if (x) cudaFree(x);
  if (e.stream) cudaStreamDestroy(e.stream);
  if (e.ev0) cudaEventDestroy(e.ev0);
  if (e.ev1) cudaEventDestroy(e.ev1);
  if (e.h_clk) cudaFreeHost(e.h_clk);
  e = Engine();
}

// The request's level-0 block tree, its rows with local neighbour slots.
void grid_rows(const shz_request& r, Grid& G) {
  const int nr = r.n / BS;
  const int nroot = nr * nr * (r.ndim == 3 ? nr : 1);
  const int bc[3] = {r.bc, r.bc, r.bc};
  shz::amr::BlockTree t(r.ndim, nr, 0, nroot, bc, bc);
  G.nblocks = nroot;
  G.rows.assign((size_t)nroot * 32, -1);
  t.table(G.rows.data());
}

// Sample the initial condition into the staging buffers, local block order; the cell numbering
// of the seeded noise is the uniform grid's, so a request starts from the state the plain
// uniform-grid step would.
void stage_uniform(const shz_server* s, Grid& G);
void stage_grid(const shz_server* s, Grid& G) {
  if (G.direct) return stage_uniform(s, G);
  const shz_request& r = G.req;
  const int n = r.n, nd = r.ndim, nr = n / BS, CB = nd == 3 ? 4096 : 256;
  shz_config c = s->cfg.hydro;
  c.n[0] = n;
  c.n[1] = n;
  c.n[2] = nd == 3 ? n : 1;
  c.dx = 1.0 / n;
  c.gamma = r.gamma;
  const shz::ProblemCtx q = shz::prepare_problem(c, r.problem);
  G.s1.resize((size_t)G.nblocks * CB);
  G.s2.resize((size_t)G.nblocks * CB);
  const double dx = 1.0 / n;
#pragma omp parallel for schedule(dynamic, 4)
  for (int b = 0; b < G.nblocks; b++) {
    const int bi = b % nr, bj = (b / nr) % nr, bk = nd == 3 ? b / (nr * nr) : 0;
    for (int t = 0; t < CB; t++) {
      const int i = bi * BS + t % BS, j = bj * BS + (t / BS) % BS, k = nd == 3 ? bk * BS + t / (BS * BS) : 0;
      const double x = (i + 0.5 - n / 2.0) * dx, y = (j + 0.5 - n / 2.0) * dx, z = nd == 3 ? (k + 0.5 - n / 2.0) * dx : 0.0;
      const uint64_t cell = ((uint64_t)k * n + j) * n + i;
      double w[6];
      shz::sample_problem(q, x, y, z, cell, w);
      const double rho = w[0], eint = w[4] / (r.gamma - 1), ke = 0.5 * rho * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
      G.s1[(size_t)b * CB + t] = make_float4((float)rho, (float)(rho * w[1]), (float)(rho * w[2]), (float)(rho * w[3]));
      G.s2[(size_t)b * CB + t] = make_float4((float)(eint + ke), (float)eint, (float)(rho * w[5]), 0.f);
    }
  }
  G.staged = true;
}

// A direct request's initial state in the uniform grid's layout (x fastest), sampled as
// stage_grid samples it.
void stage_uniform(const shz_server* s, Grid& G) {
  const shz_request& r = G.req;
  const int n = r.n, nd = r.ndim;
  shz_config c = s->cfg.hydro;
  c.n[0] = n;
  c.n[1] = n;
  c.n[2] = nd == 3 ? n : 1;
  c.dx = 1.0 / n;
  c.gamma = r.gamma;
  const shz::ProblemCtx q = shz::prepare_problem(c, r.problem);
  const size_t cells = (size_t)n * n * (nd == 3 ? n : 1);
  G.s1.resize(cells);
  G.s2.resize(cells);
  const double dx = 1.0 / n;
#pragma omp parallel for schedule(static)
  for (long long row = 0; row < (long long)n * (nd == 3 ? n : 1); row++) {
    const int j = (int)(row % n), k = (int)(row / n);
    for (int i = 0; i < n; i++) {
      const double x = (i + 0.5 - n / 2.0) * dx, y = (j + 0.5 - n / 2.0) * dx, z = nd == 3 ? (k + 0.5 - n / 2.0) * dx : 0.0;
      const uint64_t cell = ((uint64_t)k * n + j) * n + i;
      double w[6];
      shz::sample_problem(q, x, y, z, cell, w);
      const double rho = w[0], eint = w[4] / (r.gamma - 1), ke = 0.5 * rho * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
      G.s1[cell] = make_float4((float)rho, (float)(rho * w[1]), (float)(rho * w[2]), (float)(rho * w[3]));
      G.s2[cell] = make_float4((float)(eint + ke), (float)eint, (float)(rho * w[5]), 0.f);
    }
  }
  G.staged = true;
}

// Copy runs of consecutive global slots in one call each.
int upload_blocks(shz_server* s, Engine& e, Grid& G, float4* d1, float4* d2) {
  int b = 0;
  while (b < G.nblocks) {
    int run = 1;
    while (b + run < G.nblocks && G.slots[b + run] == G.slots[b] + run) run++;
    const size_t dst = (size_t)G.slots[b] * e.CB, src = (size_t)b * e.CB, cnt = (size_t)run * e.CB * sizeof(float4);
    SV_CUDA(s, cudaMemcpyAsync(d1 + dst, G.s1.data() + src, cnt, cudaMemcpyHostToDevice, e.stream));
    SV_CUDA(s, cudaMemcpyAsync(d2 + dst, G.s2.data() + src, cnt, cudaMemcpyHostToDevice, e.stream));
    b += run;
  }
  return 0;
}

// Admit a staged request: slots, parameters, clock, state.
// A direct request onto the GPU: its handle (the scheme of the server's config, the request's
// size, gamma and boundaries), its staged state uploaded.
int admit_direct(shz_server* s, Grid& G) {
  const shz_request& r = G.req;
  shz_config c = s->cfg.hydro;
  c.n[0] = r.n;
  c.n[1] = r.n;
  c.n[2] = r.ndim == 3 ? r.n : 1;
  c.dx = 1.0 / r.n;
  c.gamma = r.gamma;
  c.t_end = HUGE_VAL;
  for (int a = 0; a < 3; a++) {
    c.bc_lo[a] = a < r.ndim ? r.bc : 0;
    c.bc_hi[a] = a < r.ndim ? r.bc : 0;
  }
  c.device = s->device;
  int rc = shz_create(&c, &G.sim);
  if (rc) return fail(s, rc, "request %lld: %s", (long long)G.id, shz_last_error(nullptr));
  const size_t cells = G.s1.size();
  if ((rc = shz_set_state(G.sim, reinterpret_cast<const float*>(G.s1.data()), reinterpret_cast<const float*>(G.s2.data()),
                          cells)))
    return fail(s, rc, "request %lld: %s", (long long)G.id, shz_last_error(G.sim));
  SV_CUDA(s, cudaEventCreate(&G.ev0));
  SV_CUDA(s, cudaEventCreate(&G.ev1));
  G.s1.clear();
  G.s1.shrink_to_fit();
  G.s2.clear();
  G.s2.shrink_to_fit();
  G.enq = 0;
  s->direct_used += G.bytes;
  s->direct.push_back(&G);
  return 0;
}

// Whether the request fits what is free now.
bool fits(const shz_server* s, const Grid& G) {
  if (G.direct) return (int)s->direct.size() < DIRECT_MAX && s->direct_used + G.bytes <= s->direct_budget;
  const Engine& e = s->e[G.eng];
  return (int)e.free_slots.size() >= G.nblocks && !e.free_g.empty();
}

void release_direct(shz_server* s, Grid& G) {
  if (G.sim) {
    s->direct_launches += shz_kernel_launches(G.sim);
    shz_destroy(G.sim);
    G.sim = nullptr;
  }
  if (G.ev0) cudaEventDestroy(G.ev0);
  if (G.ev1) cudaEventDestroy(G.ev1);
  G.ev0 = G.ev1 = nullptr;
  s->direct_used -= G.bytes;
  s->direct.erase(std::find(s->direct.begin(), s->direct.end(), &G));
}

// A direct request that took its steps: its totals (and state), then its handle freed.
int finish_direct(shz_server* s, Grid& G) {
  int rc = shz_diagnostics(G.sim, &G.diag);
  if (rc) return fail(s, rc, "request %lld: %s", (long long)G.id, shz_last_error(G.sim));
  if (s->cfg.keep_states) {
    const size_t cells = (size_t)G.req.n * G.req.n * (G.req.ndim == 3 ? G.req.n : 1);
    G.out1.resize(cells * 4);
    G.out2.resize(cells * 4);
    if ((rc = shz_get_state(G.sim, G.out1.data(), G.out2.data(), cells)))
      return fail(s, rc, "request %lld: %s", (long long)G.id, shz_last_error(G.sim));
  }
  release_direct(s, G);
  G.done = true;
  G.finished = now_s(s);
  return 0;
}

int admit(shz_server* s, Grid& G) {
  if (G.direct) return admit_direct(s, G);
  Engine& e = s->e[G.eng];
  const shz_request& r = G.req;
  for (int b = 0; b < G.nblocks; b++) {
    G.slots.push_back(e.free_slots.back());
    e.free_slots.pop_back();
  }
  G.g = e.free_g.back();
  e.free_g.pop_back();
  shz::KParams P;
  std::memset(&P, 0, sizeof P);
  const shz_config& h = s->cfg.hydro;
  P.dx = 1.0 / r.n;
  P.n[0] = r.n / BS;
  P.gamma = (float)r.gamma;
  P.gm1 = (float)(r.gamma - 1);
  P.inv_gm1 = (float)(1.0 / (r.gamma - 1));
  P.inv_gamma = (float)(1.0 / r.gamma);
  P.rho_floor = (float)h.rho_floor;
  P.p_floor = (float)h.p_floor;
  P.e_floor = (float)(h.p_floor / (r.gamma - 1));
  P.eta_dual = (float)h.eta_dual;
  P.shock_thresh = (float)h.shock_thresh;
  P.signal = (float)h.signal_dims;
  P.hll = h.riemann == SHZ_RIEMANN_HLL ? 1 : 0;
  shz::DevClock c;
  std::memset(&c, 0, sizeof c);
  c.t_end = HUGE_VAL;
  c.dt_max = HUGE_VAL;
  c.cfl_dx = h.cfl;
  c.max_steps = r.steps;
  const unsigned zero[2] = {0u, 0u};
  SV_CUDA(s, cudaMemcpyAsync(e.d_gp + G.g, &P, sizeof P, cudaMemcpyHostToDevice, e.stream));
  SV_CUDA(s, cudaMemcpyAsync(e.d_clk + G.g, &c, sizeof c, cudaMemcpyHostToDevice, e.stream));
  SV_CUDA(s, cudaMemcpyAsync(e.d_rates + 2 * G.g, zero, sizeof zero, cudaMemcpyHostToDevice, e.stream));
  int rc = upload_blocks(s, e, G, e.u1[e.cur], e.u2[e.cur]);
  if (rc) return rc;
  SV_CUDA(s, cudaStreamSynchronize(e.stream));
  G.s1.clear();
  G.s1.shrink_to_fit();
  G.s2.clear();
  G.s2.shrink_to_fit();
  e.active.push_back(&G);
  e.dirty = true;
  return 0;
}

// The shared block table and work list of the running requests.
int rebuild(shz_server* s, Engine& e) {
  e.h_list.clear();
  int high = 0;
  for (Grid* G : e.active) {
    for (int b = 0; b < G->nblocks; b++) {
      const int gs = G->slots[b];
      int32_t* row = e.h_bt.data() + (size_t)gs * 32;
      const int32_t* src = G->rows.data() + (size_t)b * 32;
      for (int w = 0; w < 32; w++) row[w] = src[w];
      for (int f = 0; f < 6; f++)
        if (src[6 + f] >= 0) row[6 + f] = G->slots[src[6 + f]];
      row[26] = G->g;
      e.h_list.push_back(gs);
      high = std::max(high, gs + 1);
    }
  }
  e.high = std::max(e.high, high);
  if (e.high > 0)
    SV_CUDA(s, cudaMemcpyAsync(e.d_bt, e.h_bt.data(), (size_t)e.high * 32 * sizeof(int32_t), cudaMemcpyHostToDevice, e.stream));
  if (!e.h_list.empty())
    SV_CUDA(s, cudaMemcpyAsync(e.d_list, e.h_list.data(), e.h_list.size() * sizeof(int32_t), cudaMemcpyHostToDevice, e.stream));
  shz::amr_rest_blocks(e.h_bt.data(), e.ndim, e.h_list.data(), (int)e.h_list.size(), e.h_rest);
  if (!e.h_rest.empty())
    SV_CUDA(s, cudaMemcpyAsync(e.d_rest, e.h_rest.data(), e.h_rest.size() * sizeof(int32_t), cudaMemcpyHostToDevice, e.stream));
  e.L.rest = e.d_rest;
  e.L.nrest = (int)e.h_rest.size();
  SV_CUDA(s, cudaStreamSynchronize(e.stream));
  drop_graphs(e);
  e.dirty = false;
  return 0;
}

// One step over every running request's blocks, with the tuned launch shapes (tune_now: an eager
// step that first times the candidates of untuned kernels in place); *launches grows by the
// kernels enqueued.
int enqueue_step(shz_server* s, Engine& e, bool tune_now, long long* launches) {
  const int n = (int)e.h_list.size();
  SV_CUDA(s, shz::amr_assemble_tuned(e.L, e.d_list, n, e.u1[e.cur], e.u2[e.cur], e.d_rates, e.rslot, e.stream, tune_now,
                                     launches));
  SV_CUDA(s, shz::launch_clock_multi(e.d_clk, e.d_rates, e.rslot, e.gmax, e.stream));
  *launches += 1;
  SV_CUDA(s, shz::amr_sweep_tuned(e.L, e.d_list, n, e.u1[e.cur], e.u2[e.cur], e.u1[1 - e.cur], e.u2[1 - e.cur], e.d_clk,
                                  e.stream, tune_now, launches));
  return 0;
}

// Enqueue a round of steps (graphs, asynchronously).
int launch_round(shz_server* s, Engine& e) {
  if (e.active.empty()) return 0;
  int rc = 0;
  if (e.dirty && (rc = rebuild(s, e))) return rc;
  for (int k = 0; k < s->cfg.round_steps; k++) {
    const int nb = (int)e.h_list.size();
    if (shz::amr_step_wants_tuning(e.L, nb, nb, 0)) {
      long long c = 0;
      if ((rc = enqueue_step(s, e, true, &c))) return rc;
      e.launches += c;
      e.cur ^= 1;
      e.rslot ^= 1;
      continue;
    }
    const int gi = e.cur * 2 + e.rslot;
    cudaGraphExec_t& g = e.graphs[gi];
    if (!g) {
      cudaGraph_t graph;
      SV_CUDA(s, cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
      long long c = 0;
      rc = enqueue_step(s, e, false, &c);
      e.graph_launches[gi] = c;
      const cudaError_t ce = cudaStreamEndCapture(e.stream, &graph);
      if (rc) return rc;
      if (ce != cudaSuccess) return fail(s, SHZ_E_CUDA, "capture: %s", cudaGetErrorString(ce));
      const cudaError_t ie = cudaGraphInstantiate(&g, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) return fail(s, SHZ_E_CUDA, "instantiate: %s", cudaGetErrorString(ie));
    }
    SV_CUDA(s, cudaGraphLaunch(g, e.stream));
    e.launches += e.graph_launches[gi];
    e.cur ^= 1;
    e.rslot ^= 1;
  }
  SV_CUDA(s, cudaMemcpyAsync(e.h_clk, e.d_clk, e.gmax * sizeof(shz::DevClock), cudaMemcpyDeviceToHost, e.stream));
  return 0;
}

// A finished request: its totals (and state), then its slots back.
int finish(shz_server* s, Engine& e, Grid& G) {
  SV_CUDA(s, cudaMemcpyAsync(e.d_glist, G.slots.data(), G.nblocks * sizeof(int), cudaMemcpyHostToDevice, e.stream));
  SV_CUDA(s, shz::amr_launch_diag(e.L, e.d_glist, G.nblocks, e.u1[e.cur], e.u2[e.cur], e.d_part, e.d_out, e.stream));
  e.launches += 2;
  double v[9];
  SV_CUDA(s, cudaMemcpyAsync(v, e.d_out, sizeof v, cudaMemcpyDeviceToHost, e.stream));
  const int CB = e.CB, n = G.req.n, nd = G.req.ndim, nr = n / BS;
  std::vector<float4> b1, b2;
  if (s->cfg.keep_states) {
    b1.resize((size_t)G.nblocks * CB);
    b2.resize((size_t)G.nblocks * CB);
    for (int b = 0; b < G.nblocks; b++) {
      SV_CUDA(s, cudaMemcpyAsync(b1.data() + (size_t)b * CB, e.u1[e.cur] + (size_t)G.slots[b] * CB, CB * sizeof(float4),
                                 cudaMemcpyDeviceToHost, e.stream));
      SV_CUDA(s, cudaMemcpyAsync(b2.data() + (size_t)b * CB, e.u2[e.cur] + (size_t)G.slots[b] * CB, CB * sizeof(float4),
                                 cudaMemcpyDeviceToHost, e.stream));
    }
  }
  SV_CUDA(s, cudaStreamSynchronize(e.stream));
  const shz::DevClock& c = e.h_clk[G.g];
  G.diag.t = c.t;
  G.diag.dt = c.dt;
  G.diag.steps = c.steps;
  G.diag.mass = v[0];
  G.diag.momentum[0] = v[1];
  G.diag.momentum[1] = v[2];
  G.diag.momentum[2] = v[3];
  G.diag.e_kin = v[4];
  G.diag.e_int = v[5];
  G.diag.e_tot = v[6];
  G.diag.floored = v[7];
  G.diag.max_mach = v[8];
  if (s->cfg.keep_states) {
    const size_t cells = (size_t)n * n * (nd == 3 ? n : 1);
    G.out1.resize(cells * 4);
    G.out2.resize(cells * 4);
    for (int b = 0; b < G.nblocks; b++) {
      const int bi = b % nr, bj = (b / nr) % nr, bk = nd == 3 ? b / (nr * nr) : 0;
      for (int t = 0; t < CB; t++) {
        const int i = bi * BS + t % BS, j = bj * BS + (t / BS) % BS, k = nd == 3 ? bk * BS + t / (BS * BS) : 0;
        const size_t o = (((size_t)k * n + j) * n + i) * 4;
        const float4 a = b1[(size_t)b * CB + t], d = b2[(size_t)b * CB + t];
        G.out1[o] = a.x; G.out1[o + 1] = a.y; G.out1[o + 2] = a.z; G.out1[o + 3] = a.w;
        G.out2[o] = d.x; G.out2[o + 1] = d.y; G.out2[o + 2] = d.z; G.out2[o + 3] = d.w;
      }
    }
  }
  // idle the clock index and free the slots
  shz::DevClock idle;
  std::memset(&idle, 0, sizeof idle);
  idle.t_end = HUGE_VAL;
  idle.dt_max = HUGE_VAL;
  idle.cfl_dx = 1.0;
  SV_CUDA(s, cudaMemcpyAsync(e.d_clk + G.g, &idle, sizeof idle, cudaMemcpyHostToDevice, e.stream));
  SV_CUDA(s, cudaStreamSynchronize(e.stream));
  for (int b = G.nblocks - 1; b >= 0; b--) e.free_slots.push_back(G.slots[b]);
  e.free_g.push_back(G.g);
  G.g = -1;
  G.done = true;
  G.finished = now_s(s);
  e.active.erase(std::find(e.active.begin(), e.active.end(), &G));
  e.dirty = true;
  return 0;
}

// One round on both engines: launch, stage the queue's next requests meanwhile, then finish and
// admit.
int round_once(shz_server* s) {
  int rc = 0;
  // the direct requests' steps first, each on its handle's stream, so that they overlap the
  // batched blocks' round
  for (Grid* G : s->direct) {
    const int k = std::min(s->cfg.round_steps, G->req.steps - G->enq);
    void* sv = nullptr;
    shz_stream(G->sim, &sv);
    SV_CUDA(s, cudaEventRecord(G->ev0, static_cast<cudaStream_t>(sv)));
    if (k > 0 && (rc = shz_step(G->sim, k))) return fail(s, rc, "request %lld: %s", (long long)G->id, shz_last_error(G->sim));
    SV_CUDA(s, cudaEventRecord(G->ev1, static_cast<cudaStream_t>(sv)));
    G->enq += std::max(k, 0);
  }
  bool timed[2] = {false, false};
  for (int k = 0; k < 2; k++) {
    Engine& e = s->e[k];
    if (!e.stream || e.active.empty()) continue;
    if (!e.ev0) SV_CUDA(s, cudaEventCreate(&e.ev0));
    if (!e.ev1) SV_CUDA(s, cudaEventCreate(&e.ev1));
    SV_CUDA(s, cudaEventRecord(e.ev0, e.stream));
    if ((rc = launch_round(s, e))) return rc;
    SV_CUDA(s, cudaEventRecord(e.ev1, e.stream));
    timed[k] = true;
  }
  // stage queued requests (host work overlapping the round)
  for (Grid* G : s->pending)
    if (!G->staged) {
      stage_grid(s, *G);
      break;
    }
  for (Engine& e : s->e) {
    if (!e.stream) continue;
    SV_CUDA(s, cudaStreamSynchronize(e.stream));
    int err = 0;
    SV_CUDA(s, cudaMemcpy(&err, e.d_err, sizeof err, cudaMemcpyDeviceToHost));
    if (err) {
      cudaMemset(e.d_err, 0, sizeof(int));
      return fail(s, SHZ_E_TIMEOUT, "a kernel's bounded wait for a bulk copy ran out (code %d)", err);
    }
  }
  s->rounds++;
  float span = 0.f;
  for (int k = 0; k < 2; k++) {
    float ms = 0.f;
    if (timed[k] && cudaEventElapsedTime(&ms, s->e[k].ev0, s->e[k].ev1) == cudaSuccess) span = std::max(span, ms);
  }
  {
    std::vector<Grid*> done;
    for (Grid* G : s->direct) {
      float ms = 0.f;
      SV_CUDA(s, cudaEventSynchronize(G->ev1));
      if (cudaEventElapsedTime(&ms, G->ev0, G->ev1) == cudaSuccess) span = std::max(span, ms);
      if (G->enq >= G->req.steps) done.push_back(G);
    }
    for (Grid* G : done)
      if ((rc = finish_direct(s, *G))) return rc;
  }
  s->busy_s += span / 1000.0;
  for (Engine& e : s->e) {
    std::vector<Grid*> done;
    for (Grid* G : e.active) {
      const shz::DevClock& c = e.h_clk[G->g];
      if (c.bad) return fail(s, SHZ_E_NAN, "request %lld: the clock is NaN after %lld steps", (long long)G->id, c.steps);
      if (c.steps >= G->req.steps) done.push_back(G);
    }
    for (Grid* G : done)
      if ((rc = finish(s, e, *G))) return rc;
  }
  // admit in arrival order while the head of the queue fits
  while (!s->pending.empty()) {
    Grid* G = s->pending.front();
    if (!fits(s, *G)) break;
    if (!G->staged) stage_grid(s, *G);
    if ((rc = admit(s, *G))) return rc;
    s->pending.pop_front();
  }
  long long live = (long long)(s->e[0].active.size() + s->e[1].active.size() + s->direct.size());
  s->max_concurrent = std::max(s->max_concurrent, live);
  return 0;
}

int validate_request(const shz_server* s, const shz_request& r, std::string& why) {
  if (r.ndim != 2 && r.ndim != 3) { why = "ndim must be 2 or 3"; return -1; }
  if (r.n < BS || r.n % BS) { why = "n must be a multiple of 16"; return -1; }
  if (r.steps < 1) { why = "steps must be at least 1"; return -1; }
  if (r.bc < 0 || r.bc > 2) { why = "bc must be 0, 1 or 2"; return -1; }
  if (!(r.gamma > 1)) { why = "gamma must exceed 1"; return -1; }
  if (!shz::problem_known(r.problem.kind)) { why = "unknown problem"; return -1; }
  if (s->cfg.direct_large && direct_size(r)) {
    if (direct_bytes(r) > s->direct_budget) { why = "the request is larger than the budget for large requests"; return -1; }
    return 0;
  }
  const Engine& e = s->e[r.ndim == 3 ? 1 : 0];
  const int nr = r.n / BS;
  const int64_t nb = (int64_t)nr * nr * (r.ndim == 3 ? nr : 1);
  if (nb > e.cap) { why = "the request is larger than the whole budget"; return -1; }
  return 0;
}

Grid* enqueue(shz_server* s, const shz_request& r, double arrival) {
  auto G = std::make_unique<Grid>();
  G->id = s->next_id++;
  G->req = r;
  G->eng = r.ndim == 3 ? 1 : 0;
  G->arrival = arrival;
  G->direct = s->cfg.direct_large && direct_size(r);
  if (G->direct) G->bytes = direct_bytes(r);
  else grid_rows(r, *G);
  Grid* p = G.get();
  s->grids[p->id] = std::move(G);
  s->pending.push_back(p);
  return p;
}

void fill_stats(const std::vector<Grid*>& gs, double t_first, long long rounds, long long maxc, long long launches,
                double busy_s, shz_server_stats* out) {
  std::vector<double> lat;
  double zu = 0, last = t_first;
  for (const Grid* G : gs) {
    lat.push_back(G->finished - G->arrival);
    last = std::max(last, G->finished);
    zu += std::pow((double)G->req.n, G->req.ndim) * G->req.steps;
  }
  std::sort(lat.begin(), lat.end());
  auto q = [&](double p) {
    if (lat.empty()) return 0.0;
    const double x = p * (lat.size() - 1);
    const size_t i = (size_t)x;
    const double f = x - i;
    return i + 1 < lat.size() ? lat[i] * (1 - f) + lat[i + 1] * f : lat[i];
  };
  double mean = 0;
  for (double v : lat) mean += v;
  out->completed = (int64_t)gs.size();
  out->makespan_s = last - t_first;
  out->p50_s = q(0.5);
  out->p99_s = q(0.99);
  out->mean_s = lat.empty() ? 0 : mean / lat.size();
  out->zone_updates = zu;
  out->zu_per_s = out->makespan_s > 0 ? zu / out->makespan_s : 0;
  out->max_concurrent = maxc;
  out->rounds = rounds;
  out->kernel_launches = launches;
  out->busy_s = busy_s;
}

}  // namespace

extern "C" {

const char* shz_server_error(const shz_server* s) { return s ? s->err.c_str() : g_create_err.c_str(); }

int shz_server_create(const shz_server_config* cfg, shz_server** out) {
  if (!cfg || !out) return SHZ_E_CONFIG;
  *out = nullptr;
  if (cfg->max_grids < 1 || cfg->round_steps < 1 || !(cfg->budget_bytes > 0)) {
    g_create_err = "refused server configuration: max_grids, round_steps and budget_bytes must be positive";
    return SHZ_E_CONFIG;
  }
  if (cfg->hydro.recon < 0 || cfg->hydro.recon > SHZ_RECON_KOREN) {
    g_create_err = "refused server configuration: the block passes take minmod, mc, vanleer or koren";
    return SHZ_E_CONFIG;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    g_create_err = "no CUDA device";
    return SHZ_E_NODEV;
  }
  Dev dv(cfg->hydro.device);
  shz_server* s = new shz_server();
  s->cfg = *cfg;
  s->device = cfg->hydro.device;
  // a sixth of the budget for 2D requests, the rest for 3D; with direct_large a quarter of it is
  // kept for the large requests' uniform grids, the rest split so
  const double blocks_budget = cfg->direct_large ? cfg->budget_bytes * 0.75 : cfg->budget_bytes;
  s->direct_budget = cfg->direct_large ? cfg->budget_bytes * 0.25 : 0.0;
  int rc = engine_init(s, s->e[0], 2, blocks_budget / 6.0);
  if (!rc) rc = engine_init(s, s->e[1], 3, blocks_budget * 5.0 / 6.0);
  if (rc) {
    g_create_err = s->err;
    shz_server_destroy(s);
    return rc;
  }
  *out = s;
  return SHZ_OK;
}

void shz_server_destroy(shz_server* s) {
  if (!s) return;
  Dev dv(s->device);
  while (!s->direct.empty()) release_direct(s, *s->direct.back());
  for (Engine& e : s->e) engine_free(e);
  delete s;
}

int shz_server_submit(shz_server* s, const shz_request* r, int64_t* id) {
  if (!s || !r) return SHZ_E_CONFIG;
  std::string why;
  if (validate_request(s, *r, why)) return fail(s, SHZ_E_CONFIG, "refused request: %s", why.c_str());
  Grid* G = enqueue(s, *r, now_s(s));
  if (id) *id = G->id;
  return 0;
}

int shz_server_drain(shz_server* s, int32_t max_rounds) {
  if (!s) return SHZ_E_CONFIG;
  Dev dv(s->device);
  int rounds = 0;
  while (!s->pending.empty() || running(s)) {
    if (!running(s)) {
      // nothing running: admit the head of the queue
      Grid* G = s->pending.front();
      if (!G->staged) stage_grid(s, *G);
      int rc = admit(s, *G);
      if (rc) return rc;
      s->pending.pop_front();
      continue;
    }
    int rc = round_once(s);
    if (rc) return rc;
    if (max_rounds > 0 && ++rounds >= max_rounds) break;
  }
  return 0;
}

int shz_server_run_stream(shz_server* s, const shz_request* reqs, int32_t n, shz_server_stats* out) {
  if (!s || (!reqs && n) || !out) return SHZ_E_CONFIG;
  Dev dv(s->device);
  for (int i = 0; i < n; i++) {
    std::string why;
    if (validate_request(s, reqs[i], why)) return fail(s, SHZ_E_CONFIG, "refused request %d: %s", i, why.c_str());
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return reqs[a].arrival < reqs[b].arrival; });
  const double base = now_s(s);
  const long long r0 = s->rounds;
  const double busy0 = s->busy_s;
  long long l0 = s->e[0].launches + s->e[1].launches + s->direct_launches;
  s->max_concurrent = 0;
  std::vector<Grid*> mine;
  size_t next = 0;
  while (next < order.size() || !s->pending.empty() || running(s)) {
    const double t = now_s(s) - base;
    while (next < order.size() && reqs[order[next]].arrival <= t) {
      mine.push_back(enqueue(s, reqs[order[next]], base + reqs[order[next]].arrival));
      next++;
    }
    if (!running(s)) {
      if (!s->pending.empty()) {
        Grid* G = s->pending.front();
        if (!G->staged) stage_grid(s, *G);
        int rc = admit(s, *G);
        if (rc) return rc;
        s->pending.pop_front();
        continue;
      }
      if (next < order.size()) {
        const double wait = reqs[order[next]].arrival - (now_s(s) - base);
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
      }
      continue;
    }
    int rc = round_once(s);
    if (rc) return rc;
  }
  fill_stats(mine, base + (n ? reqs[order[0]].arrival : 0.0), s->rounds - r0, s->max_concurrent,
             s->e[0].launches + s->e[1].launches + s->direct_launches - l0, s->busy_s - busy0, out);
  return 0;
}

int shz_server_cancel(shz_server* s, int64_t id) {
  if (!s) return SHZ_E_CONFIG;
  auto it = s->grids.find(id);
  if (it == s->grids.end()) return fail(s, SHZ_E_CONFIG, "no request %lld", (long long)id);
  Grid& G = *it->second;
  if (G.done) return fail(s, SHZ_E_CONFIG, "request %lld has %s", (long long)id, G.cancelled ? "been cancelled" : "finished");
  Dev dv(s->device);
  auto q = std::find(s->pending.begin(), s->pending.end(), &G);
  if (q != s->pending.end()) {
    s->pending.erase(q);
    G.s1.clear();
    G.s1.shrink_to_fit();
    G.s2.clear();
    G.s2.shrink_to_fit();
  } else if (G.direct) {
    release_direct(s, G);  // its handle's work is done between calls: freed at once
  } else {
    // admitted: no round is in flight between calls, so its slots and clock go back at once
    Engine& e = s->e[G.eng];
    shz::DevClock idle;
    std::memset(&idle, 0, sizeof idle);
    idle.t_end = HUGE_VAL;
    idle.dt_max = HUGE_VAL;
    idle.cfl_dx = 1.0;
    SV_CUDA(s, cudaMemcpyAsync(e.d_clk + G.g, &idle, sizeof idle, cudaMemcpyHostToDevice, e.stream));
    SV_CUDA(s, cudaStreamSynchronize(e.stream));
    for (int b = G.nblocks - 1; b >= 0; b--) e.free_slots.push_back(G.slots[b]);
    e.free_g.push_back(G.g);
    G.g = -1;
    e.active.erase(std::find(e.active.begin(), e.active.end(), &G));
    e.dirty = true;
  }
  G.cancelled = true;
  G.done = true;
  G.finished = now_s(s);
  return 0;
}

int shz_server_poll(shz_server* s, int64_t id, int32_t* status, int64_t* steps_done) {
  if (!s || !status) return SHZ_E_CONFIG;
  auto it = s->grids.find(id);
  if (it == s->grids.end()) return fail(s, SHZ_E_CONFIG, "no request %lld", (long long)id);
  const Grid& G = *it->second;
  int64_t done = 0;
  if (G.cancelled) {
    *status = SHZ_REQ_CANCELLED;
  } else if (G.done) {
    *status = SHZ_REQ_FINISHED;
    done = G.req.steps;
  } else if (std::find(s->pending.begin(), s->pending.end(), &G) != s->pending.end()) {
    *status = SHZ_REQ_QUEUED;
  } else {
    *status = SHZ_REQ_RUNNING;
    // between calls no round is in flight: the clocks read back after the last round are current
    done = G.direct ? G.enq : (G.g >= 0 ? s->e[G.eng].h_clk[G.g].steps : 0);
  }
  if (steps_done) *steps_done = done;
  return 0;
}

int shz_server_result(shz_server* s, int64_t id, shz_diag* d) {
  if (!s || !d) return SHZ_E_CONFIG;
  auto it = s->grids.find(id);
  if (it == s->grids.end()) return fail(s, SHZ_E_CONFIG, "no request %lld", (long long)id);
  if (it->second->cancelled) return fail(s, SHZ_E_CANCELLED, "request %lld was cancelled", (long long)id);
  if (!it->second->done) return fail(s, SHZ_E_CONFIG, "request %lld has not finished", (long long)id);
  *d = it->second->diag;
  return 0;
}

int shz_server_state(shz_server* s, int64_t id, float* u1, float* u2) {
  if (!s || !u1 || !u2) return SHZ_E_CONFIG;
  auto it = s->grids.find(id);
  if (it != s->grids.end() && it->second->cancelled)
    return fail(s, SHZ_E_CANCELLED, "request %lld was cancelled", (long long)id);
  if (it == s->grids.end() || !it->second->done) return fail(s, SHZ_E_CONFIG, "request %lld has not finished", (long long)id);
  if (it->second->out1.empty()) return fail(s, SHZ_E_CONFIG, "states are kept only with keep_states");
  std::memcpy(u1, it->second->out1.data(), it->second->out1.size() * sizeof(float));
  std::memcpy(u2, it->second->out2.data(), it->second->out2.size() * sizeof(float));
  return 0;
}

int shz_plain_run_stream(const shz_server_config* cfg, const shz_request* reqs, int32_t n, shz_server_stats* out) {
  if (!cfg || (!reqs && n) || !out) return SHZ_E_CONFIG;
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return reqs[a].arrival < reqs[b].arrival; });
  const auto t0 = Clock::now();
  auto now = [&]() { return std::chrono::duration<double>(Clock::now() - t0).count(); };
  std::vector<std::unique_ptr<Grid>> gs;
  std::vector<Grid*> ptrs;
  long long launches = 0;
  double busy = 0;
  for (int i : order) {
    const shz_request& r = reqs[i];
    const double wait = r.arrival - now();
    if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
    shz_config c = cfg->hydro;
    c.n[0] = r.n;
    c.n[1] = r.n;
    c.n[2] = r.ndim == 3 ? r.n : 1;
    c.dx = 1.0 / r.n;
    c.gamma = r.gamma;
    for (int a = 0; a < 3; a++) {
      c.bc_lo[a] = a < r.ndim ? r.bc : 0;
      c.bc_hi[a] = a < r.ndim ? r.bc : 0;
    }
    shz_sim* sim = nullptr;
    int rc = shz_create(&c, &sim);
    if (rc) return rc;
    if ((rc = shz_reset_problem(sim, &r.problem))) {
      shz_destroy(sim);
      return rc;
    }
    shz_run_opts o{r.steps, std::numeric_limits<double>::quiet_NaN(), 0.0};
    shz_run_result res;
    // the run's span on the handle's stream: the GPU-busy part of this request
    void* sv = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const bool timed = shz_stream(sim, &sv) == 0 && cudaEventCreate(&e0) == cudaSuccess &&
                       cudaEventCreate(&e1) == cudaSuccess;
    if (timed) cudaEventRecord(e0, static_cast<cudaStream_t>(sv));
    rc = shz_run(sim, &o, &res);
    if (timed) {
      cudaEventRecord(e1, static_cast<cudaStream_t>(sv));
      float ms = 0.f;
      if (cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) busy += ms / 1000.0;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    launches += shz_kernel_launches(sim);
    shz_destroy(sim);
    if (rc) return rc;
    auto G = std::make_unique<Grid>();
    G->req = r;
    G->arrival = r.arrival;
    G->finished = now();
    ptrs.push_back(G.get());
    gs.push_back(std::move(G));
  }
  fill_stats(ptrs, n ? reqs[order[0]].arrival : 0.0, 0, 1, launches, busy, out);
  return 0;
}

}  // extern "C"
