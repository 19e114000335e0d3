// The adaptive-grid run (shz_amr_*): the host side of the reference's AmrSim
// (src/amr/amr_sim.ts). It owns the block tree (amr_tree.cpp), the atlases in HBM, the block
// table and slot lists on the device, and one stream. A step is one CUDA graph of three or four
// kernels (assemble, clock, the matched faces' fine fluxes where the mesh has any, the fused block
// sweep: amr_kernels.cu), or of four with two_pass (predict and update in place of the last two);
// every regrid_every steps the Löhner flags
// are read back, BlockTree.adapt decides the new mesh on the host, the new tables go up and the
// regrid kernel fills the new leaves (amr_sim.ts:2648 applyRegrid, :3033 encodeFlags, :3525 readFlags);
// the check runs at the start of the next step, from that step's own assemble (check_step).
// With per-block timesteps (time_bins) time advances in cycles of 2^time_bins substeps
// (amr_sim.ts:1509-1660 encodeCycle): see cycle_once.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/shaderous_b200.h"
#include "amr_kernels.h"
#include "amr_tree.h"
#include "problems.h"
#include "sweep.h"

using shz::amr::BlockTree;
using shz::amr::RegridOp;

struct shz_amr {
  shz_amr_config cfg;
  shz::AmrLaunch L;
  std::unique_ptr<BlockTree> tree;
  int CB = 0, WN = 0, PN = 0;
  float4* u1[2] = {nullptr, nullptr};
  float4* u2[2] = {nullptr, nullptr};
  float4 *w1 = nullptr, *w2 = nullptr, *p1 = nullptr, *p2 = nullptr;
  int *d_bt = nullptr, *d_all = nullptr, *d_leaves = nullptr, *d_rg = nullptr;
  shz::KParams* d_gp = nullptr;  // this run's parameters: grid 0 of the passes' per-grid table
  float* d_flags = nullptr;
  shz::DevClock* clk = nullptr;
  shz::DevClock* clk_save = nullptr;  // the clock before a step taken ahead of its refinement check
  cudaEvent_t flags_ready = nullptr;
  unsigned* rates = nullptr;  // slots 0, 1: the steps'; 2, 3: the refinement check's
  double *diag_part = nullptr, *diag_out = nullptr;
  int* d_ghost = nullptr;
  int* d_err = nullptr;  // the kernels' error word
  // faces matched to refined neighbours (fused sweep): (leaf slot, face, entry) triples and the
  // buffer of their mean fine fluxes, grown with the mesh
  int* d_flist = nullptr;
  int* d_rest = nullptr;  // the split assemble's second-pass blocks (amr_rest_blocks)
  std::vector<int32_t> h_rest;
  float4* fbuf = nullptr;
  int nfine = 0, fine_cap = 0;
  std::vector<int32_t> h_bt, h_all, h_leaves, h_rg, h_flist;
  std::vector<float> h_flags;
  float* h_flags_pinned = nullptr;  // the refinement check's flags, copied back while the step runs
  int cur = 0, slot = 0;
  long long since_check = 0;
  // a refinement check is due before the next single step: its assemble is that step's own
  bool flags_due = false;
  // whether the next check takes its step ahead of the decision: after a check that kept the mesh
  // (a step taken ahead of a check that changes it is thrown away)
  bool check_ahead = true;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graphs[4] = {nullptr, nullptr, nullptr, nullptr};
  long long graph_launches[4] = {0, 0, 0, 0};  // kernels one replay of each graph launches
  long long launches = 0;
  std::string err;
  int device = 0;
  // Per-block timesteps: the bin tables (the relaxation's two buffers; [0] the substep, [1 + slot]
  // the bin), each leaf's own rate / dx from the cycle's first assemble, the substeps' block lists
  // (built on the host from the bins), and the bookkeeping of pauses and work (amr_sim.ts:437-445).
  int* d_bins[2] = {nullptr, nullptr};
  float* d_brate = nullptr;
  int* d_cyc = nullptr;
  int32_t* h_cyc = nullptr;   // pinned: the lists of a cycle's substeps, uploaded in one copy
  int32_t* h_bins = nullptr;  // pinned: the bin table read back at the start of each cycle
  size_t cyc_cap = 0;
  cudaEvent_t bins_ready = nullptr;
  int bin_pause = 0, bin_pause_next = 0, cycles_since_poll = 0;
  long long bin_cycles = 0, bin_updates = 0, bin_single = 0, seen_updates = 0, seen_single = 0;
};

namespace {

int fail(shz_amr* a, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (a) a->err = buf;
  return code;
}

std::string g_create_err;

#define AMR_CUDA(a, call)                                                                                 \
  do {                                                                                                    \
    cudaError_t e_ = (call);                                                                              \
    if (e_ != cudaSuccess)                                                                                \
      return fail(a, e_ == cudaErrorMemoryAllocation ? SHZ_E_OOM : SHZ_E_CUDA, "%s: %s", #call,          \
                  cudaGetErrorString(e_));                                                                \
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

void drop_graphs(shz_amr* a) {
  for (auto& g : a->graphs)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

// The fine-flux buffer and its face list for at least `faces` matched faces (grown with the mesh).
int grow_fbuf(shz_amr* a, int faces) {
  if (faces <= a->fine_cap) return 0;
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  cudaFree(a->d_flist);
  cudaFree(a->fbuf);
  a->d_flist = nullptr;
  a->fbuf = nullptr;
  a->fine_cap = 0;
  const int want = faces + faces / 2 + 64;
  const size_t fc = a->cfg.ndim == 3 ? 256 : 16;
  if (cudaMalloc(&a->d_flist, (size_t)want * 3 * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&a->fbuf, (size_t)want * fc * 2 * sizeof(float4)) != cudaSuccess) {
    cudaGetLastError();
    return fail(a, SHZ_E_OOM, "the fine-flux buffer of %d matched faces does not fit", want);
  }
  a->fine_cap = want;
  a->L.fbuf = a->fbuf;
  // (the single steps' list of faces matched to refined neighbours moves with the buffer, and the
  // steps' graphs captured the old addresses)
  if (!a->h_flist.empty())
    AMR_CUDA(a, cudaMemcpyAsync(a->d_flist, a->h_flist.data(), a->h_flist.size() * sizeof(int32_t),
                                cudaMemcpyHostToDevice, a->stream));
  drop_graphs(a);
  return 0;
}

// The block table and the slot lists of the current tree, to the device.
int upload_tables(shz_amr* a) {
  const int cap = a->cfg.cap;
  a->h_bt.resize((size_t)cap * shz::amr::BT_STRIDE);
  a->tree->table(a->h_bt.data());
  for (int s = 0; s < cap; s++) a->h_bt[(size_t)s * shz::amr::BT_STRIDE + 26] = 0;  // every block is grid 0's
  std::vector<int32_t> per;
  a->tree->lists(a->h_all, a->h_leaves, per);
  // the fused sweep's matched faces: each leaf's faces whose same-level neighbour is refined get
  // consecutive buffer entries, the first in word 27 of its row
  a->h_flist.clear();
  if (!a->cfg.two_pass) {
    const int32_t* bt = a->h_bt.data();
    const int S = shz::amr::BT_STRIDE;
    for (int s : a->h_leaves) {
      for (int f = 0; f < 2 * a->cfg.ndim; f++) {
        const int nb = bt[(size_t)s * S + 6 + f];
        if (nb < 0 || (bt[(size_t)nb * S + 4] & 2)) continue;
        const int k = (int)(a->h_flist.size() / 3);
        if (a->h_bt[(size_t)s * S + 27] < 0) a->h_bt[(size_t)s * S + 27] = k;
        a->h_flist.insert(a->h_flist.end(), {s, f, k});
      }
    }
  }
  a->nfine = (int)(a->h_flist.size() / 3);
  int rc = grow_fbuf(a, a->nfine);
  if (rc) return rc;
  a->L.err = a->d_err;
  if (a->nfine > 0)
    AMR_CUDA(a, cudaMemcpyAsync(a->d_flist, a->h_flist.data(), a->h_flist.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                a->stream));
  AMR_CUDA(a, cudaMemcpyAsync(a->d_bt, a->h_bt.data(), a->h_bt.size() * sizeof(int32_t), cudaMemcpyHostToDevice, a->stream));
  AMR_CUDA(a, cudaMemcpyAsync(a->d_all, a->h_all.data(), a->h_all.size() * sizeof(int32_t), cudaMemcpyHostToDevice, a->stream));
  AMR_CUDA(a, cudaMemcpyAsync(a->d_leaves, a->h_leaves.data(), a->h_leaves.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                              a->stream));
  // the blocks of the assemble's list with ghosts beyond a level change (the split assemble's rest)
  const std::vector<int32_t>& asm_list = a->cfg.two_pass ? a->h_all : a->h_leaves;
  shz::amr_rest_blocks(a->h_bt.data(), a->cfg.ndim, asm_list.data(), (int)asm_list.size(), a->h_rest);
  if (!a->h_rest.empty())
    AMR_CUDA(a, cudaMemcpyAsync(a->d_rest, a->h_rest.data(), a->h_rest.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                a->stream));
  a->L.rest = a->d_rest;
  a->L.nrest = (int)a->h_rest.size();
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  drop_graphs(a);
  return 0;
}

// The kernels' error word: a bounded wait inside a kernel that ran out (tma::ERR_*) fails the call.
int check_err(shz_amr* a) {
  int e = 0;
  AMR_CUDA(a, cudaMemcpyAsync(&e, a->d_err, sizeof e, cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  if (e) {
    cudaMemsetAsync(a->d_err, 0, sizeof(int), a->stream);
    return fail(a, SHZ_E_TIMEOUT, "a kernel's bounded wait for a bulk copy ran out (code %d); the state is not valid", e);
  }
  return 0;
}

int read_clock(shz_amr* a, shz::DevClock* h) {
  AMR_CUDA(a, cudaMemcpyAsync(h, a->clk, sizeof *h, cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  return check_err(a);
}

int write_clock(shz_amr* a, double t, long long steps) {
  shz::DevClock h;
  std::memset(&h, 0, sizeof h);
  h.t = t;
  h.t_end = a->cfg.hydro.t_end;
  h.dt_max = a->cfg.hydro.dt_max;
  h.cfl_dx = a->cfg.hydro.cfl;  // the rates are per unit of each block's own cell size
  h.steps = steps;
  h.max_steps = std::numeric_limits<long long>::max();
  AMR_CUDA(a, cudaMemcpyAsync(a->clk, &h, sizeof h, cudaMemcpyHostToDevice, a->stream));
  AMR_CUDA(a, cudaMemsetAsync(a->rates, 0, 4 * sizeof(unsigned), a->stream));
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  return 0;
}


int n_all(const shz_amr* a) { return (int)a->h_all.size(); }
int n_leaves(const shz_amr* a) { return (int)a->h_leaves.size(); }

// One step's kernels, enqueued with the tuned launch shapes; *launches grows by the kernels
// enqueued. With tune_now (an eager step, never a capture), kernels whose shape is not tuned yet
// are timed in place over their candidates first (each candidate repeats the same step's work);
// the clock is read back so that a held step (which only copies) tunes nothing.
// The assemble of a step (its first kernel).
int enqueue_assemble(shz_amr* a, bool tune_now, long long* launches) {
  // (the two passes predict same-level ghosts at their source, whose atlas may be a parent's;
  // everything the fused sweep reads is a leaf's)
  const int* asm_list = a->cfg.two_pass ? a->d_all : a->d_leaves;
  const int asm_n = a->cfg.two_pass ? n_all(a) : n_leaves(a);
  AMR_CUDA(a, shz::amr_assemble_tuned(a->L, asm_list, asm_n, a->u1[a->cur], a->u2[a->cur], a->rates, a->slot, a->stream,
                                      tune_now, launches));
  return 0;
}

// The rest of a step after its assemble: the clock, then the fine-flux pass and the sweep (or the
// two passes).
int enqueue_rest(shz_amr* a, bool tune_now, long long* launches) {
  AMR_CUDA(a, shz::launch_clock_multi(a->clk, a->rates, a->slot, 1, a->stream));
  *launches += 1;
  if (tune_now) {
    shz::DevClock h;
    int rc = read_clock(a, &h);
    if (rc) return rc;
    tune_now = !h.held;
  }
  if (a->cfg.two_pass) {
    AMR_CUDA(a, shz::amr_launch_predict(a->L, a->d_leaves, n_leaves(a), a->clk, a->stream));
    AMR_CUDA(a, shz::amr_launch_update(a->L, a->d_leaves, n_leaves(a), a->u1[a->cur], a->u2[a->cur], a->u1[1 - a->cur],
                                       a->u2[1 - a->cur], a->clk, a->stream));
    *launches += 2;
  } else {
    AMR_CUDA(a, shz::amr_fine_flux_tuned(a->L, a->d_flist, a->nfine, a->clk, a->stream, tune_now, launches));
    AMR_CUDA(a, shz::amr_sweep_tuned(a->L, a->d_leaves, n_leaves(a), a->u1[a->cur], a->u2[a->cur], a->u1[1 - a->cur],
                                     a->u2[1 - a->cur], a->clk, a->stream, tune_now, launches));
  }
  return 0;
}

int enqueue_step(shz_amr* a, bool tune_now, long long* launches) {
  int rc = enqueue_assemble(a, tune_now, launches);
  return rc ? rc : enqueue_rest(a, tune_now, launches);
}

// One step, as the CUDA graph of its kernels for this (state parity, rate slot); the graphs
// are captured once per mesh and replayed.
int step_once(shz_amr* a) {
  // a mesh whose kernels meet a size class the tuner has not seen: one eager step that tunes
  if (!a->cfg.two_pass &&
      shz::amr_step_wants_tuning(a->L, n_leaves(a), n_leaves(a), a->nfine)) {
    long long n = 0;
    const int rc = enqueue_step(a, true, &n);
    if (rc) return rc;
    a->launches += n;
    a->cur ^= 1;
    a->slot ^= 1;
    return 0;
  }
  const int gi = a->cur * 2 + a->slot;
  cudaGraphExec_t& g = a->graphs[gi];
  if (!g) {
    cudaGraph_t graph;
    AMR_CUDA(a, cudaStreamBeginCapture(a->stream, cudaStreamCaptureModeThreadLocal));
    long long n = 0;
    int rc = enqueue_step(a, false, &n);
    cudaError_t e = cudaStreamEndCapture(a->stream, &graph);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(a, SHZ_E_CUDA, "capture of a step: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&g, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(a, SHZ_E_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    a->graph_launches[gi] = n;
  }
  AMR_CUDA(a, cudaGraphLaunch(g, a->stream));
  a->launches += a->graph_launches[gi];
  a->cur ^= 1;
  a->slot ^= 1;
  return 0;
}

// Per-block timesteps' pauses (amr_sim.ts:136-151): a run's first single steps, the polls of the
// cycles' share of block updates, the share above which they pause, and the pauses.
constexpr int BIN_START_STEPS = 16;
constexpr int BIN_POLL_CYCLES = 4;
constexpr double BIN_SHARE_MAX = 0.8;
constexpr int BIN_PAUSE_STEPS = 192;
constexpr int BIN_PAUSE_MAX = 1536;

void reset_bins(shz_amr* a) {
  a->bin_pause = a->cfg.time_bins > 0 ? BIN_START_STEPS : 0;
  a->bin_pause_next = BIN_PAUSE_STEPS;
  a->cycles_since_poll = 0;
  a->bin_cycles = a->bin_updates = a->bin_single = a->seen_updates = a->seen_single = 0;
}

// Whether leaf `slot` has a face neighbour in a faster bin than its own: a same-level leaf, or a
// child of a refined same-level neighbour that touches the shared face (amr/bins_lists.wgsl:27-51).
bool faster_neighbor(const shz_amr* a, const int32_t* kb, int slot) {
  const int S = shz::amr::BT_STRIDE;
  const int32_t* bt = a->h_bt.data();
  const int k = kb[1 + slot];
  for (int f = 0; f < 2 * a->cfg.ndim; f++) {
    const int nb = bt[(size_t)slot * S + 6 + f];
    if (nb < 0 || nb == slot) continue;
    if (bt[(size_t)nb * S + 4] & 2) {
      if (kb[1 + nb] < k) return true;
      continue;
    }
    // refined: its children on the shared face (beyond our lower face, its upper children)
    const int axis = f >> 1, want = 1 - (f & 1);
    for (int ch = 0; ch < 8; ch++) {
      if (((ch >> axis) & 1) != want) continue;
      const int c = bt[(size_t)nb * S + 12 + ch];
      if (c >= 0 && (bt[(size_t)c * S + 4] & 2) && kb[1 + c] < k) return true;
    }
  }
  return false;
}

// One cycle of per-block timesteps (amr_sim.ts:1509-1660 encodeCycle): 2^K substeps of the
// clock's dt, after which every block is at the same time again.
//   substep 0: every block steps. The assemble measures each leaf's rate; the clock sets the
//     cycle's dt (short enough for the cycle to end by the stop time); the bins follow from the
//     rates (first guess, dilation, relaxation); then predict and update, each block with its own
//     step 2^k dt, and with its faster neighbours' fluxes through the shared faces for half of it.
//   substeps s = 1 .. 2^K - 1: the blocks that start a step (s a multiple of 2^k) are assembled,
//     the leaves among them predicted, and updated together with the leaves half way through their
//     step that have a faster neighbour (the deposit of its second-step fluxes).
// The bin table is read back once per cycle (while substep 0's passes run) and the substeps'
// lists are built here, in the order of the block list (amr/bins_lists.wgsl gathers them with
// atomics in no fixed order; no result depends on it). The state stays in one parity: the update
// writes in place.
void after_cycle(shz_amr* a, long long updates, int nl);

int cycle_two(shz_amr* a) {
  const int K = a->cfg.time_bins, n = 1 << K;
  float4* u1 = a->u1[a->cur];
  float4* u2 = a->u2[a->cur];
  int* A = a->d_bins[0];
  int* B = a->d_bins[1];
  const int na = n_all(a), nl = n_leaves(a);
  unsigned* scratch = a->rates + 4;  // the later substeps' assembles: rates nothing reads
  AMR_CUDA(a, shz::amr_launch_bins_tick(a->clk, A, 0, a->stream));
  AMR_CUDA(a, shz::amr_assemble_bins_tuned(a->L, a->d_all, na, u1, u2, A, a->rates, a->slot, a->d_brate, a->stream, &a->launches));
  AMR_CUDA(a, shz::launch_clock_multi(a->clk, a->rates, a->slot, 1, a->stream, n));
  const int sweeps = (K + a->cfg.max_level + 2) | 1;
  AMR_CUDA(a, shz::amr_launch_bins(a->L, a->d_all, na, a->d_brate, a->clk, (float)a->cfg.hydro.cfl, K, sweeps, A, B,
                                   a->stream));
  AMR_CUDA(a, cudaMemcpyAsync(a->h_bins, A, (size_t)(a->cfg.cap + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaMemcpyAsync(a->h_bins + a->cfg.cap + 1, &a->clk->held, sizeof(int), cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaEventRecord(a->bins_ready, a->stream));
  AMR_CUDA(a, shz::amr_launch_predict(a->L, a->d_leaves, nl, a->clk, a->stream, A));
  AMR_CUDA(a, shz::amr_launch_update(a->L, a->d_leaves, nl, u1, u2, u1, u2, a->clk, a->stream, A));
  a->launches += 7 + sweeps;
  a->slot ^= 1;
  AMR_CUDA(a, cudaEventSynchronize(a->bins_ready));
  if (a->h_bins[a->cfg.cap + 1]) return 0;  // a held cycle: nothing to step
  // the substeps' lists: per substep the counts of LA (assembled), LL (predicted), LU (updated),
  // then the three lists
  const size_t per = 3 + (size_t)na + 2 * (size_t)nl;
  const size_t need = (size_t)(n - 1) * per;
  if (need > a->cyc_cap) {
    cudaFree(a->d_cyc);
    cudaFreeHost(a->h_cyc);
    a->d_cyc = nullptr;
    a->h_cyc = nullptr;
    a->cyc_cap = 0;
    if (cudaMalloc(&a->d_cyc, need * sizeof(int32_t)) != cudaSuccess ||
        cudaMallocHost(&a->h_cyc, need * sizeof(int32_t)) != cudaSuccess) {
      cudaGetLastError();
      return fail(a, SHZ_E_OOM, "the block lists of a cycle (%zu ints) do not fit", need);
    }
    a->cyc_cap = need;
  }
  const int32_t* kb = a->h_bins;
  const int32_t* bt = a->h_bt.data();
  const int S = shz::amr::BT_STRIDE;
  long long updates = nl;
  for (int sub = 1; sub < n; sub++) {
    int32_t* rec = a->h_cyc + (size_t)(sub - 1) * per;
    int32_t* la = rec + 3;
    int32_t* ll = la + na;
    int32_t* lu = ll + nl;
    int ca = 0, cl = 0, cu = 0;
    for (int slot : a->h_all) {
      const int k = kb[1 + slot];
      const int phase = sub & ((1 << k) - 1);
      const bool on = phase == 0;
      const bool leaf = (bt[(size_t)slot * S + 4] & 2) != 0;
      if (on) la[ca++] = slot;
      if (on && leaf) ll[cl++] = slot;
      const bool deposit = leaf && !on && k > 0 && phase == (1 << (k - 1)) && faster_neighbor(a, kb, slot);
      if (leaf && (on || deposit)) lu[cu++] = slot;
    }
    rec[0] = ca;
    rec[1] = cl;
    rec[2] = cu;
    updates += cu;
  }
  AMR_CUDA(a, cudaMemcpyAsync(a->d_cyc, a->h_cyc, need * sizeof(int32_t), cudaMemcpyHostToDevice, a->stream));
  for (int sub = 1; sub < n; sub++) {
    const int32_t* rec = a->h_cyc + (size_t)(sub - 1) * per;
    const int* la = a->d_cyc + (size_t)(sub - 1) * per + 3;
    const int* ll = la + na;
    const int* lu = ll + nl;
    AMR_CUDA(a, shz::amr_launch_bins_tick(a->clk, A, sub, a->stream));
    AMR_CUDA(a, shz::amr_assemble_bins_tuned(a->L, la, rec[0], u1, u2, A, scratch, 0, nullptr, a->stream, &a->launches));
    AMR_CUDA(a, shz::amr_launch_predict(a->L, ll, rec[1], a->clk, a->stream, A));
    AMR_CUDA(a, shz::amr_launch_update(a->L, lu, rec[2], u1, u2, u1, u2, a->clk, a->stream, A));
    a->launches += 1 + (rec[0] > 0) + (rec[1] > 0) + (rec[2] > 0);
  }
  after_cycle(a, updates, nl);
  return 0;
}

// The work of a cycle, and a poll every few cycles: above the share, single steps for a while,
// longer each time (amr_sim.ts:2992-3020 pollBins).
void after_cycle(shz_amr* a, long long updates, int nl) {
  a->bin_cycles++;
  a->bin_updates += updates;
  a->bin_single += (long long)nl << a->cfg.time_bins;
  if (++a->cycles_since_poll >= BIN_POLL_CYCLES) {
    a->cycles_since_poll = 0;
    const long long du = a->bin_updates - a->seen_updates, ds = a->bin_single - a->seen_single;
    a->seen_updates = a->bin_updates;
    a->seen_single = a->bin_single;
    if (ds > 0 && !a->cfg.time_bins_always) {
      if ((double)du / (double)ds > BIN_SHARE_MAX) {
        a->bin_pause = a->bin_pause_next;
        a->bin_pause_next = std::min(BIN_PAUSE_MAX, 2 * a->bin_pause_next);
      } else {
        a->bin_pause_next = BIN_PAUSE_STEPS;
      }
    }
  }
}

// The fused form of a cycle: as cycle_two, with the fused sweep over the leaves that start a step,
// and ahead of it, per substep, the neighbour-flux pass over the faces of the leaves that update
// whose neighbour is refined or a faster leaf; then the deposits of the leaves half way through
// their step beside a faster neighbour. Only leaves are assembled (the sweep and the flux pass
// read leaves' atlases alone). The bin table is read back before substep 0's sweep, whose faces
// already depend on the bins.
int cycle_fused(shz_amr* a) {
  const int K = a->cfg.time_bins, n = 1 << K;
  float4* u1 = a->u1[a->cur];
  float4* u2 = a->u2[a->cur];
  int* A = a->d_bins[0];
  int* B = a->d_bins[1];
  const int na = n_all(a), nl = n_leaves(a), cap = a->cfg.cap;
  unsigned* scratch = a->rates + 4;
  AMR_CUDA(a, shz::amr_launch_bins_tick(a->clk, A, 0, a->stream));
  AMR_CUDA(a, shz::amr_assemble_bins_tuned(a->L, a->d_leaves, nl, u1, u2, A, a->rates, a->slot, a->d_brate, a->stream, &a->launches));
  AMR_CUDA(a, shz::launch_clock_multi(a->clk, a->rates, a->slot, 1, a->stream, n));
  const int sweeps = (K + a->cfg.max_level + 2) | 1;
  AMR_CUDA(a, shz::amr_launch_bins(a->L, a->d_all, na, a->d_brate, a->clk, (float)a->cfg.hydro.cfl, K, sweeps, A, B,
                                   a->stream));
  AMR_CUDA(a, cudaMemcpyAsync(a->h_bins, A, (size_t)(cap + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaMemcpyAsync(a->h_bins + cap + 1, &a->clk->held, sizeof(int), cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaEventRecord(a->bins_ready, a->stream));
  a->launches += 5 + sweeps;
  a->slot ^= 1;
  AMR_CUDA(a, cudaEventSynchronize(a->bins_ready));
  if (a->h_bins[cap + 1]) return 0;  // a held cycle: nothing to step
  // per substep: the leaves that start a step (swept), those that take a deposit, the faces whose
  // fluxes come from the neighbour-flux pass (slot, face, entry), and each slot's first entry
  const int32_t* kb = a->h_bins;
  const int32_t* bt = a->h_bt.data();
  const int S = shz::amr::BT_STRIDE;
  const int nf = 2 * a->cfg.ndim;
  struct Sub {
    size_t ll, ld, e, fb;
    int nll, nld, ne;
  };
  std::vector<Sub> subs(n);
  std::vector<int32_t> buf;
  buf.reserve((size_t)n * (2 * (size_t)nl + cap));
  long long updates = 0;
  int most = 0;
  for (int sub = 0; sub < n; sub++) {
    Sub& q = subs[sub];
    std::vector<int32_t> ld, ents;
    q.ll = buf.size();
    for (int slot : a->h_leaves) {
      const int k = kb[1 + slot];
      const int phase = sub & ((1 << k) - 1);
      if (phase == 0) buf.push_back(slot);
      else if (k > 0 && phase == (1 << (k - 1)) && faster_neighbor(a, kb, slot)) ld.push_back(slot);
    }
    q.nll = (int)(buf.size() - q.ll);
    q.ld = buf.size();
    buf.insert(buf.end(), ld.begin(), ld.end());
    q.nld = (int)ld.size();
    q.fb = buf.size();
    buf.resize(buf.size() + cap, -1);
    int ne = 0;
    auto faces_of = [&](int slot) {
      const int k = kb[1 + slot];
      for (int f = 0; f < nf; f++) {
        const int nb = bt[(size_t)slot * S + 6 + f];
        if (nb < 0) continue;
        const bool leaf = (bt[(size_t)nb * S + 4] & 2) != 0;
        if (leaf && (nb == slot || kb[1 + nb] >= k)) continue;
        if (buf[q.fb + slot] < 0) buf[q.fb + slot] = ne;
        ents.insert(ents.end(), {slot, f, ne});
        ne++;
      }
    };
    for (size_t i = q.ll; i < q.ll + q.nll; i++) faces_of(buf[i]);
    for (int slot : ld) faces_of(slot);
    q.e = buf.size();
    buf.insert(buf.end(), ents.begin(), ents.end());
    q.ne = ne;
    most = std::max(most, ne);
    updates += q.nll + q.nld;
  }
  int rc = grow_fbuf(a, most);
  if (rc) return rc;
  if (buf.size() > a->cyc_cap) {
    AMR_CUDA(a, cudaStreamSynchronize(a->stream));
    cudaFree(a->d_cyc);
    cudaFreeHost(a->h_cyc);
    a->d_cyc = nullptr;
    a->h_cyc = nullptr;
    a->cyc_cap = 0;
    const size_t want = buf.size() + buf.size() / 4;
    if (cudaMalloc(&a->d_cyc, want * sizeof(int32_t)) != cudaSuccess ||
        cudaMallocHost(&a->h_cyc, want * sizeof(int32_t)) != cudaSuccess) {
      cudaGetLastError();
      return fail(a, SHZ_E_OOM, "the block lists of a cycle (%zu ints) do not fit", want);
    }
    a->cyc_cap = want;
  }
  std::memcpy(a->h_cyc, buf.data(), buf.size() * sizeof(int32_t));
  AMR_CUDA(a, cudaMemcpyAsync(a->d_cyc, a->h_cyc, buf.size() * sizeof(int32_t), cudaMemcpyHostToDevice, a->stream));
  shz::AmrLaunch L = a->L;
  L.bins = A;
  for (int sub = 0; sub < n; sub++) {
    const Sub& q = subs[sub];
    const int* ll = a->d_cyc + q.ll;
    L.fbase = a->d_cyc + q.fb;
    if (sub > 0) {
      AMR_CUDA(a, shz::amr_launch_bins_tick(a->clk, A, sub, a->stream));
      AMR_CUDA(a, shz::amr_assemble_bins_tuned(L, ll, q.nll, u1, u2, A, scratch, 0, nullptr, a->stream, &a->launches));
      a->launches += 1 + (q.nll > 0);
    }
    AMR_CUDA(a, shz::amr_launch_fine_flux(L, a->d_cyc + q.e, q.ne, a->clk, a->stream));
    AMR_CUDA(a, shz::amr_launch_sweep(L, ll, q.nll, u1, u2, u1, u2, a->clk, a->stream));
    AMR_CUDA(a, shz::amr_launch_deposit(L, a->d_cyc + q.ld, q.nld, u1, u2, a->clk, a->stream));
    a->launches += (q.ne > 0) + (q.nll > 0) + (q.nld > 0);
  }
  after_cycle(a, updates, nl);
  return 0;
}

int cycle_once(shz_amr* a) { return a->cfg.two_pass ? cycle_two(a) : cycle_fused(a); }

// The refinement indicators of the current state: a fresh assemble, then the Löhner pass.
int compute_flags(shz_amr* a) {
  AMR_CUDA(a, cudaMemsetAsync(a->rates + 2, 0, 2 * sizeof(unsigned), a->stream));
  long long n = 0;
  AMR_CUDA(a, shz::amr_assemble_tuned(a->L, a->cfg.two_pass ? a->d_all : a->d_leaves,
                                      a->cfg.two_pass ? n_all(a) : n_leaves(a), a->u1[a->cur], a->u2[a->cur],
                                      a->rates + 2, 0, a->stream, false, &n));
  AMR_CUDA(a, cudaMemsetAsync(a->d_flags, 0, sizeof(float) * a->cfg.cap, a->stream));
  AMR_CUDA(a, shz::amr_launch_flag(a->L, a->d_leaves, n_leaves(a), a->d_flags, a->stream));
  a->launches += 2;
  a->h_flags.resize(a->cfg.cap);
  AMR_CUDA(a, cudaMemcpyAsync(a->h_flags.data(), a->d_flags, sizeof(float) * a->cfg.cap, cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  return 0;
}

// tree.adapt over the indicators; if the mesh changed, the new tables and the regrid pass.
int check_and_regrid(shz_amr* a, const std::vector<double>* extra, int* changed) {
  int rc = compute_flags(a);
  if (rc) return rc;
  std::vector<RegridOp> ops;
  try {
    ops = a->tree->adapt(
        [&](const shz::amr::Block* b) {
          double v = a->h_flags[b->slot];
          if (extra) v = std::max(v, (*extra)[b->slot]);
          return v;
        },
        a->cfg.refine_hi, a->cfg.refine_lo);
  } catch (const std::exception& e) {
    return fail(a, SHZ_E_CONFIG, "adapt: %s", e.what());
  }
  *changed = ops.empty() ? 0 : 1;
  if (ops.empty()) return 0;
  a->h_rg.resize((size_t)a->cfg.cap * shz::amr::RG_STRIDE);
  BlockTree::regrid_table(ops, a->cfg.cap, a->h_rg.data());
  AMR_CUDA(a, cudaMemcpyAsync(a->d_rg, a->h_rg.data(), a->h_rg.size() * sizeof(int32_t), cudaMemcpyHostToDevice, a->stream));
  if ((rc = upload_tables(a))) return rc;
  if (!extra) {
    AMR_CUDA(a, shz::amr_launch_regrid(a->L, a->d_rg, a->d_leaves, n_leaves(a), a->u1[a->cur], a->u2[a->cur],
                                       a->u1[1 - a->cur], a->u2[1 - a->cur], a->stream));
    a->launches += 1;
    a->cur ^= 1;
  }
  return 0;
}

// A single step that begins with the refinement check due after the last (amr_sim.ts applies a
// re-mesh decided after a step at the start of the next, applyRegrid): the step's own assemble
// gives the primitives the Löhner pass reads, so the check needs no assemble of its own. After a
// check that kept the mesh, the rest of the step is launched at once, ahead of the decision (the
// reference's speculation behind an unanswered check, amr_sim.ts:2762-2775), and BlockTree.adapt
// runs on the host meanwhile. The step writes the other parity, so the state it started from is
// still there: if the mesh changes, the clock is put back as it was, the new leaves are filled from
// that state and the step runs again on the new mesh (its rate taken back); if not, the step
// stands. After a check that changed the mesh (a moving front changes it at check after check),
// the rest waits for the decision: the host's adapt is a few milliseconds, a step thrown away
// several times that. Either way the same kernels run on the same data. Launched eagerly, not from
// a graph.
int check_step(shz_amr* a) {
  a->flags_due = false;
  const bool ahead = a->check_ahead;
  long long n = 0;
  int rc = enqueue_assemble(a, false, &n);
  if (rc) return rc;
  AMR_CUDA(a, cudaMemsetAsync(a->d_flags, 0, sizeof(float) * a->cfg.cap, a->stream));
  AMR_CUDA(a, shz::amr_launch_flag(a->L, a->d_leaves, n_leaves(a), a->d_flags, a->stream));
  n += 1;
  a->h_flags.resize(a->cfg.cap);
  AMR_CUDA(a, cudaMemcpyAsync(a->h_flags_pinned, a->d_flags, sizeof(float) * a->cfg.cap, cudaMemcpyDeviceToHost,
                              a->stream));
  AMR_CUDA(a, cudaEventRecord(a->flags_ready, a->stream));
  if (ahead) {
    AMR_CUDA(a, cudaMemcpyAsync(a->clk_save, a->clk, sizeof(shz::DevClock), cudaMemcpyDeviceToDevice, a->stream));
    if ((rc = enqueue_rest(a, false, &n))) return rc;
  }
  a->launches += n;
  AMR_CUDA(a, cudaEventSynchronize(a->flags_ready));
  std::memcpy(a->h_flags.data(), a->h_flags_pinned, sizeof(float) * a->cfg.cap);
  std::vector<RegridOp> ops;
  try {
    ops = a->tree->adapt([&](const shz::amr::Block* b) { return (double)a->h_flags[b->slot]; }, a->cfg.refine_hi,
                         a->cfg.refine_lo);
  } catch (const std::exception& e) {
    return fail(a, SHZ_E_CONFIG, "adapt: %s", e.what());
  }
  a->check_ahead = ops.empty();
  if (!ops.empty()) {
    // the step taken ahead (if any) is void: the clock as it was; the rate slot, which the
    // assemble filled over the old mesh, empty for the new one
    if (ahead)
      AMR_CUDA(a, cudaMemcpyAsync(a->clk, a->clk_save, sizeof(shz::DevClock), cudaMemcpyDeviceToDevice, a->stream));
    AMR_CUDA(a, cudaMemsetAsync(a->rates + a->slot, 0, sizeof(unsigned), a->stream));
    a->h_rg.resize((size_t)a->cfg.cap * shz::amr::RG_STRIDE);
    BlockTree::regrid_table(ops, a->cfg.cap, a->h_rg.data());
    AMR_CUDA(a, cudaMemcpyAsync(a->d_rg, a->h_rg.data(), a->h_rg.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                                a->stream));
    if ((rc = upload_tables(a))) return rc;
    AMR_CUDA(a, shz::amr_launch_regrid(a->L, a->d_rg, a->d_leaves, n_leaves(a), a->u1[a->cur], a->u2[a->cur],
                                       a->u1[1 - a->cur], a->u2[1 - a->cur], a->stream));
    a->launches += 1;
    a->cur ^= 1;
    return step_once(a);
  }
  if (!ahead) {
    n = 0;
    if ((rc = enqueue_rest(a, false, &n))) return rc;
    a->launches += n;
  }
  a->cur ^= 1;
  a->slot ^= 1;
  return 0;
}

// Level-0 cell size and the finest grid, for sampling problems.
double dx0_of(const shz_amr_config& c) { return c.box / (c.nr * shz::amr::BS); }

shz_config fine_config(const shz_amr_config& c) {
  shz_config f = c.hydro;
  const int nf = (c.nr * shz::amr::BS) << c.max_level;
  f.n[0] = nf;
  f.n[1] = c.ndim >= 2 ? nf : 1;
  f.n[2] = c.ndim == 3 ? nf : 1;
  f.dx = c.box / nf;
  return f;
}

// Whether a problem's discontinuity crosses a block's box (the initial mesh refines there even
// where no cell centre of a coarse block sees it).
bool crosses(const shz::ProblemCtx& q, const double lo[3], const double hi[3], int nd) {
  const shz_problem& p = q.p;
  auto sphere = [&](double r) {
    double d2 = 0, far2 = 0;
    for (int a = 0; a < nd; a++) {
      const double c = std::min(std::max(0.0, lo[a]), hi[a]);
      d2 += c * c;
      const double f = std::max(std::fabs(lo[a]), std::fabs(hi[a]));
      far2 += f * f;
    }
    return d2 <= r * r && far2 >= r * r;
  };
  switch (p.kind) {
    case SHZ_PROB_SOD: return lo[p.axis] <= 0 && hi[p.axis] >= 0;
    case SHZ_PROB_SEDOV: return sphere(q.sedov_r);
    case SHZ_PROB_BLAST: return sphere(p.a[4]);
    case SHZ_PROB_KH: {
      const double e = 0.25 * q.L[1];
      return (lo[1] <= e && hi[1] >= e) || (lo[1] <= -e && hi[1] >= -e);
    }
    default: return false;
  }
}

// Sample the problem into every leaf, and upload (u[cur]).
int sample_leaves(shz_amr* a, const shz::ProblemCtx& q) {
  const int BS = shz::amr::BS, nd = a->cfg.ndim, CB = a->CB;
  const double dx0 = dx0_of(a->cfg), half = a->cfg.box / 2;
  const int batch = 256;
  float4 *h1 = nullptr, *h2 = nullptr;
  AMR_CUDA(a, cudaMallocHost(&h1, (size_t)batch * CB * sizeof(float4)));
  if (cudaMallocHost(&h2, (size_t)batch * CB * sizeof(float4)) != cudaSuccess) {
    cudaFreeHost(h1);
    return fail(a, SHZ_E_OOM, "pinned staging");
  }
  int rc = 0;
  const int nl = n_leaves(a);
  for (int b0 = 0; b0 < nl && rc == 0; b0 += batch) {
    const int b1 = std::min(nl, b0 + batch);
#pragma omp parallel for schedule(dynamic)
    for (int bi = b0; bi < b1; bi++) {
      const int slot = a->h_leaves[bi];
      const int32_t* row = a->h_bt.data() + (size_t)slot * shz::amr::BT_STRIDE;
      const int lev = row[0];
      const double dx = dx0 / (double)(1 << lev);
      const uint64_t span = (uint64_t)(a->cfg.nr * BS) << lev;
      for (int t = 0; t < CB; t++) {
        const int i = t % BS, j = (t / BS) % BS, k = nd == 3 ? t / (BS * BS) : 0;
        const int gi = row[1] * BS + i, gj = row[2] * BS + j, gk = nd == 3 ? row[3] * BS + k : 0;
        const double x = (gi + 0.5) * dx - half, y = (gj + 0.5) * dx - half, z = nd == 3 ? (gk + 0.5) * dx - half : 0.0;
        const uint64_t cell = ((((uint64_t)lev << 56) ^ ((uint64_t)gk * span + gj)) * span) + gi;
        double w[6];
        shz::sample_problem(q, x, y, z, cell, w);
        const double rho = w[0], eint = w[4] / (a->cfg.hydro.gamma - 1);
        const double ke = 0.5 * rho * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
        const size_t o = (size_t)(bi - b0) * CB + t;
        h1[o] = make_float4((float)rho, (float)(rho * w[1]), (float)(rho * w[2]), (float)(rho * w[3]));
        h2[o] = make_float4((float)(eint + ke), (float)eint, (float)(rho * w[5]), 0.f);
      }
    }
    for (int bi = b0; bi < b1 && rc == 0; bi++) {
      const size_t dst = (size_t)a->h_leaves[bi] * CB, src = (size_t)(bi - b0) * CB;
      if (cudaMemcpyAsync(a->u1[a->cur] + dst, h1 + src, CB * sizeof(float4), cudaMemcpyHostToDevice, a->stream) != cudaSuccess ||
          cudaMemcpyAsync(a->u2[a->cur] + dst, h2 + src, CB * sizeof(float4), cudaMemcpyHostToDevice, a->stream) != cudaSuccess)
        rc = fail(a, SHZ_E_CUDA, "leaf upload");
    }
    if (cudaStreamSynchronize(a->stream) != cudaSuccess) rc = fail(a, SHZ_E_CUDA, "leaf upload sync");
  }
  cudaFreeHost(h1);
  cudaFreeHost(h2);
  return rc;
}

// n steps (substeps of whole cycles with per-block timesteps, which may run past n); *taken: the
// steps taken.
int step_n(shz_amr* a, int n, int* taken) {
  int i = 0;
  while (i < n) {
    // with per-block timesteps, whole cycles (which may run past n), unless paused
    const bool cycle = a->cfg.time_bins > 0 && a->bin_pause == 0;
    if (!cycle && a->bin_pause > 0) a->bin_pause--;
    int rc = 0;
    if (cycle && a->flags_due) {
      // the mesh is checked between cycles, before the next begins
      a->flags_due = false;
      int changed = 0;
      if ((rc = check_and_regrid(a, nullptr, &changed))) return rc;
    }
    rc = cycle ? cycle_once(a) : a->flags_due ? check_step(a) : step_once(a);
    if (rc) return rc;
    const int took = cycle ? 1 << a->cfg.time_bins : 1;
    i += took;
    a->since_check += took;
    if (a->cfg.regrid_every > 0 && a->since_check >= a->cfg.regrid_every) {
      a->since_check = 0;
      a->flags_due = true;
    }
  }
  if (taken) *taken = i;
  return 0;
}

}  // namespace

extern "C" {

const char* shz_amr_error(const shz_amr* a) { return a ? a->err.c_str() : g_create_err.c_str(); }

int shz_amr_create(const shz_amr_config* cfg, shz_amr** out) {
  if (!cfg || !out) return SHZ_E_CONFIG;
  *out = nullptr;
  const shz_amr_config& c = *cfg;
  auto refuse = [&](const char* why) {
    g_create_err = std::string("refused AMR configuration: ") + why;
    return SHZ_E_CONFIG;
  };
  if (c.ndim != 2 && c.ndim != 3) return refuse("ndim must be 2 or 3");
  if (c.nr < 1 || c.max_level < 0 || c.max_level > shz::amr::MAX_LEVELS) return refuse("nr >= 1 and max_level 0..7");
  if (c.hydro.recon == SHZ_RECON_PPM) return refuse("PPM reaches three cells; the blocks keep two ghost layers");
  if (c.time_bins < 0 || c.time_bins > 5) return refuse("time_bins is 0 (off) to 5 (cycles of 32 substeps)");
  if (c.hydro.recon < 0 || c.hydro.recon > SHZ_RECON_KOREN) return refuse("recon must be minmod, mc, vanleer or koren");
  if (!(c.box > 0) || !(c.hydro.gamma > 1) || !(c.hydro.cfl > 0)) return refuse("box > 0, gamma > 1, cfl > 0");
  for (int ax = 0; ax < 3; ax++)
    if (c.hydro.bc_lo[ax] < 0 || c.hydro.bc_lo[ax] > 2 || c.hydro.bc_hi[ax] < 0 || c.hydro.bc_hi[ax] > 2)
      return refuse("boundary codes are 0, 1, 2");
  const int nroot = c.nr * c.nr * (c.ndim == 3 ? c.nr : 1);
  if (c.cap < nroot) return refuse("cap is smaller than the root blocks");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    g_create_err = "no CUDA device";
    return SHZ_E_NODEV;
  }
  if (c.hydro.device < 0 || c.hydro.device >= count) return refuse("no such device");
  Dev dv(c.hydro.device);
  shz_amr* a = new shz_amr();
  a->cfg = c;
  a->device = c.hydro.device;
  a->CB = c.ndim == 3 ? 4096 : 256;
  a->WN = c.ndim == 3 ? 8000 : 400;
  a->PN = c.ndim == 3 ? 5832 : 324;
  shz::KParams P;
  std::memset(&P, 0, sizeof P);
  P.dx = dx0_of(c);
  P.n[0] = c.nr;
  P.gamma = (float)c.hydro.gamma;
  P.gm1 = (float)(c.hydro.gamma - 1);
  P.inv_gm1 = (float)(1.0 / (c.hydro.gamma - 1));
  P.inv_gamma = (float)(1.0 / c.hydro.gamma);
  P.rho_floor = (float)c.hydro.rho_floor;
  P.p_floor = (float)c.hydro.p_floor;
  P.e_floor = (float)(c.hydro.p_floor / (c.hydro.gamma - 1));
  P.eta_dual = (float)c.hydro.eta_dual;
  P.shock_thresh = (float)c.hydro.shock_thresh;
  P.signal = (float)c.hydro.signal_dims;
  P.hll = c.hydro.riemann == SHZ_RIEMANN_HLL ? 1 : 0;
  a->L.ndim = c.ndim;
  a->L.recon = c.hydro.recon;
  a->L.isen = c.hydro.isentropic != 0;
  a->L.per_texel = a->cfg.two_pass != 0;
  auto bail = [&](int code, const char* what) {
    g_create_err = what;
    shz_amr_destroy(a);
    return code;
  };
  const size_t cap = c.cap;
  if (cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(SHZ_E_CUDA, "stream");
  if (cudaStreamCreateWithFlags(&a->L.side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&a->L.fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&a->L.join, cudaEventDisableTiming) != cudaSuccess)
    return bail(SHZ_E_CUDA, "side stream");
  bool ok = true;
  for (int p = 0; p < 2; p++) {
    ok = ok && cudaMalloc(&a->u1[p], cap * a->CB * sizeof(float4)) == cudaSuccess;
    ok = ok && cudaMalloc(&a->u2[p], cap * a->CB * sizeof(float4)) == cudaSuccess;
  }
  ok = ok && cudaMalloc(&a->w1, cap * a->WN * sizeof(float4)) == cudaSuccess;
  ok = ok && cudaMalloc(&a->w2, cap * a->WN * sizeof(float4)) == cudaSuccess;
  if (a->cfg.two_pass || c.time_bins > 0) {
    ok = ok && cudaMalloc(&a->p1, cap * a->PN * sizeof(float4)) == cudaSuccess;
    ok = ok && cudaMalloc(&a->p2, cap * a->PN * sizeof(float4)) == cudaSuccess;
  }
  ok = ok && cudaMalloc(&a->d_bt, cap * shz::amr::BT_STRIDE * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc(&a->d_all, cap * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc(&a->d_leaves, cap * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc(&a->d_rest, cap * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc(&a->d_rg, cap * shz::amr::RG_STRIDE * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc(&a->d_flags, cap * sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&a->clk, sizeof(shz::DevClock)) == cudaSuccess;
  ok = ok && cudaMalloc(&a->clk_save, sizeof(shz::DevClock)) == cudaSuccess;
  ok = ok && cudaMallocHost(&a->h_flags_pinned, cap * sizeof(float)) == cudaSuccess;
  ok = ok && cudaEventCreateWithFlags(&a->flags_ready, cudaEventDisableTiming) == cudaSuccess;
  ok = ok && cudaMalloc(&a->rates, 6 * sizeof(unsigned)) == cudaSuccess;
  if (ok) ok = cudaMemset(a->rates, 0, 6 * sizeof(unsigned)) == cudaSuccess;
  if (c.time_bins > 0) {
    for (int p = 0; p < 2; p++) {
      ok = ok && cudaMalloc(&a->d_bins[p], (cap + 1) * sizeof(int)) == cudaSuccess;
      if (ok) ok = cudaMemset(a->d_bins[p], 0, (cap + 1) * sizeof(int)) == cudaSuccess;
    }
    ok = ok && cudaMalloc(&a->d_brate, cap * sizeof(float)) == cudaSuccess;
    if (ok) ok = cudaMemset(a->d_brate, 0, cap * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMallocHost(&a->h_bins, (cap + 2) * sizeof(int32_t)) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&a->bins_ready, cudaEventDisableTiming) == cudaSuccess;
  }
  ok = ok && cudaMalloc(&a->d_gp, sizeof(shz::KParams)) == cudaSuccess;
  // (room for the 9 totals or the 13 extended channels per block)
  ok = ok && cudaMalloc(&a->diag_part, (size_t)shz::amr_diag_blocks(c.cap) * 16 * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&a->diag_out, 16 * sizeof(double)) == cudaSuccess;
  ok = ok && cudaMalloc(&a->d_ghost, (size_t)a->WN * 5 * sizeof(int)) == cudaSuccess;
  ok = ok && cudaMalloc(&a->d_err, sizeof(int)) == cudaSuccess;
  if (ok) ok = cudaMemset(a->d_err, 0, sizeof(int)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    char buf[160];
    snprintf(buf, sizeof buf, "the atlases of %d block slots (%.2f GB) do not fit", c.cap,
             cap * (4.0 * a->CB + 2.0 * a->WN + (a->L.p1 || a->cfg.two_pass || c.time_bins > 0 ? 2.0 * a->PN : 0.0)) * 16 / 1e9);
    return bail(SHZ_E_OOM, buf);
  }
  a->L.bt = a->d_bt;
  a->L.gp = a->d_gp;
  if (cudaMemcpy(a->d_gp, &P, sizeof P, cudaMemcpyHostToDevice) != cudaSuccess) return bail(SHZ_E_CUDA, "parameters upload");
  a->L.w1 = a->w1;
  a->L.w2 = a->w2;
  a->L.p1 = a->p1;
  a->L.p2 = a->p2;
  // the tree of root blocks, a quiet uniform state, the clock at 0
  try {
    a->tree.reset(new BlockTree(c.ndim, c.nr, c.max_level, c.cap, c.hydro.bc_lo, c.hydro.bc_hi));
  } catch (const std::exception& e) {
    return bail(SHZ_E_CONFIG, e.what());
  }
  if (upload_tables(a) || write_clock(a, 0.0, 0)) return bail(SHZ_E_CUDA, a->err.c_str());
  reset_bins(a);
  *out = a;
  return SHZ_OK;
}

void shz_amr_destroy(shz_amr* a) {
  if (!a) return;
  Dev dv(a->device);
  if (a->stream) cudaStreamSynchronize(a->stream);
  drop_graphs(a);
  for (int p = 0; p < 2; p++) {
    cudaFree(a->u1[p]);
    cudaFree(a->u2[p]);
  }
  void* bufs[] = {a->w1, a->w2, a->p1, a->p2, a->d_bt, a->d_all, a->d_leaves, a->d_rg, a->d_flags, a->d_gp,
                  a->clk, a->rates, a->diag_part, a->diag_out, a->d_ghost, a->d_flist, a->fbuf, a->d_err,
                  a->d_bins[0], a->d_bins[1], a->d_brate, a->d_cyc, a->clk_save, a->d_rest};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (a->h_bins) cudaFreeHost(a->h_bins);
  if (a->h_flags_pinned) cudaFreeHost(a->h_flags_pinned);
  if (a->flags_ready) cudaEventDestroy(a->flags_ready);
  if (a->h_cyc) cudaFreeHost(a->h_cyc);
  if (a->bins_ready) cudaEventDestroy(a->bins_ready);
  if (a->stream) cudaStreamDestroy(a->stream);
  if (a->L.fork) cudaEventDestroy(a->L.fork);
  if (a->L.join) cudaEventDestroy(a->L.join);
  if (a->L.side) cudaStreamDestroy(a->L.side);
  delete a;
}

int shz_amr_reset_problem(shz_amr* a, const shz_problem* prob) {
  if (!a || !prob) return SHZ_E_CONFIG;
  if (!shz::problem_known(prob->kind)) return fail(a, SHZ_E_CONFIG, "unknown problem kind %d", prob->kind);
  Dev dv(a->device);
  const shz_amr_config& c = a->cfg;
  try {
    a->tree.reset(new BlockTree(c.ndim, c.nr, c.max_level, c.cap, c.hydro.bc_lo, c.hydro.bc_hi));
  } catch (const std::exception& e) {
    return fail(a, SHZ_E_CONFIG, "%s", e.what());
  }
  int rc = upload_tables(a);
  if (rc) return rc;
  a->cur = 0;
  a->slot = 0;
  const shz::ProblemCtx q = shz::prepare_problem(fine_config(c), *prob);
  const double dx0 = dx0_of(c), half = c.box / 2;
  // The initial mesh: adapt over the sampled state, each pass re-sampling every leaf.
  for (int pass = 0; pass <= c.max_level; pass++) {
    if ((rc = sample_leaves(a, q))) return rc;
    if (pass == c.max_level) break;
    std::vector<double> feature(c.cap, 0.0);
    for (int s : a->h_leaves) {
      const int32_t* row = a->h_bt.data() + (size_t)s * shz::amr::BT_STRIDE;
      const double side = dx0 / (double)(1 << row[0]) * shz::amr::BS;
      double lo[3], hi[3];
      for (int ax = 0; ax < 3; ax++) {
        lo[ax] = row[1 + ax] * side - half;
        hi[ax] = lo[ax] + side;
      }
      if (crosses(q, lo, hi, c.ndim)) feature[s] = 2.0 * c.refine_hi + 1.0;
    }
    int changed = 0;
    if ((rc = check_and_regrid(a, &feature, &changed))) return rc;
    if (!changed) break;
  }
  a->since_check = 0;
  a->flags_due = false;
  reset_bins(a);
  return write_clock(a, 0.0, 0);
}

int shz_amr_step(shz_amr* a, int32_t n) {
  if (!a || n < 0) return SHZ_E_CONFIG;
  Dev dv(a->device);
  return step_n(a, n, nullptr);
}

int shz_amr_regrid(shz_amr* a, int32_t* changed) {
  if (!a || !changed) return SHZ_E_CONFIG;
  Dev dv(a->device);
  int ch = 0;
  a->flags_due = false;
  int rc = check_and_regrid(a, nullptr, &ch);
  *changed = ch;
  return rc;
}

int shz_amr_clock(shz_amr* a, double* t, double* dt, int64_t* steps) {
  if (!a) return SHZ_E_CONFIG;
  Dev dv(a->device);
  shz::DevClock h;
  int rc = read_clock(a, &h);
  if (rc) return rc;
  if (t) *t = h.t;
  if (dt) *dt = h.dt;
  if (steps) *steps = h.steps;
  if (h.bad) return fail(a, SHZ_E_NAN, "the clock is NaN after %lld steps", h.steps);
  return 0;
}

int shz_amr_run(shz_amr* a, const shz_run_opts* o, shz_run_result* r) {
  if (!a || !o || !r) return SHZ_E_CONFIG;
  Dev dv(a->device);
  const auto t0 = std::chrono::steady_clock::now();
  auto ms = [&]() { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); };
  const bool has_until = !std::isnan(o->until);
  if (o->steps < 0 && !has_until) return fail(a, SHZ_E_CONFIG, "run() needs `steps`, `until`, or both");
  shz::DevClock c;
  int rc = read_clock(a, &c);
  if (rc) return rc;
  const long long start = c.steps;
  double last_dt = c.last_dt;
  const double t_end_was = a->cfg.hydro.t_end;
  const double stop = has_until ? std::min(o->until, t_end_was) : t_end_was;
  if (stop != t_end_was) AMR_CUDA(a, cudaMemcpyAsync(&a->clk->t_end, &stop, sizeof(double), cudaMemcpyHostToDevice, a->stream));
  int stopped = SHZ_STOP_STEPS;
  int grow = 1;
  double ms_per_step = 0;  // the batches' pace
  for (;;) {
    const long long taken = c.steps - start;
    const long long left = o->steps < 0 ? std::numeric_limits<long long>::max() : o->steps - taken;
    if (left <= 0) { stopped = SHZ_STOP_STEPS; break; }
    if (has_until && c.t >= o->until * (1 - 1e-12)) { stopped = SHZ_STOP_TIME; break; }
    if (std::isfinite(t_end_was) && c.t >= t_end_was * (1 - 1e-12)) { stopped = SHZ_STOP_END; break; }
    if (o->timeout_ms > 0 && ms() > o->timeout_ms) { stopped = SHZ_STOP_TIMEOUT; break; }
    long long batch = std::min<long long>(left, grow);
    // batches of about 100 ms on blocks (api.ts run: BATCH_MS for an adaptive mesh)
    if (ms_per_step > 0) batch = std::min<long long>(batch, std::max(1.0, std::floor(100.0 / ms_per_step)));
    if (std::isfinite(stop) && last_dt > 0) {
      const double ahead = std::ceil((stop - c.t) / last_dt - 1e-6);
      if (ahead >= 1 && ahead < (double)batch) batch = (long long)ahead;
    }
    batch = std::max<long long>(batch, 1);
    const double b0 = ms();
    if ((rc = shz_amr_step(a, (int)batch))) break;
    if ((rc = read_clock(a, &c))) break;
    if (c.bad) { rc = fail(a, SHZ_E_NAN, "the clock is NaN after %lld steps", c.steps); break; }
    if (c.last_dt > 0) last_dt = c.last_dt;
    if (c.steps - start == taken) {
      stopped = has_until && c.t >= o->until * (1 - 1e-9) ? SHZ_STOP_TIME : SHZ_STOP_END;
      break;
    }
    const double m = (ms() - b0) / (double)batch;
    ms_per_step = ms_per_step > 0 ? 0.7 * ms_per_step + 0.3 * m : m;
    grow = std::min(grow * 2, 64);
  }
  if (stop != t_end_was) {
    cudaMemcpyAsync(&a->clk->t_end, &t_end_was, sizeof(double), cudaMemcpyHostToDevice, a->stream);
    cudaStreamSynchronize(a->stream);
  }
  if (rc) return rc;
  r->t = c.t;
  r->dt = c.dt;
  r->steps = c.steps;
  r->taken = c.steps - start;
  r->seconds = ms() / 1000.0;
  r->stopped = stopped;
  r->last_dt = last_dt;
  return 0;
}

int shz_amr_diagnostics(shz_amr* a, shz_diag* d) {
  if (!a || !d) return SHZ_E_CONFIG;
  Dev dv(a->device);
  AMR_CUDA(a, shz::amr_launch_diag(a->L, a->d_leaves, n_leaves(a), a->u1[a->cur], a->u2[a->cur], a->diag_part, a->diag_out,
                                   a->stream));
  a->launches += 2;
  double v[9];
  AMR_CUDA(a, cudaMemcpyAsync(v, a->diag_out, sizeof v, cudaMemcpyDeviceToHost, a->stream));
  shz::DevClock c;
  int rc = read_clock(a, &c);
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

int shz_amr_diagnostics_ext(shz_amr* a, shz_diag_ext* d) {
  if (!a || !d) return SHZ_E_CONFIG;
  int rc = shz_amr_diagnostics(a, &d->base);
  if (rc) return rc;
  Dev dv(a->device);
  AMR_CUDA(a, shz::amr_launch_diag_ext(a->L, a->d_leaves, n_leaves(a), a->u1[a->cur], a->u2[a->cur], a->diag_part,
                                       a->diag_out, a->stream));
  a->launches += 2;
  double v[shz::DIAG_EXT_VALUES];
  AMR_CUDA(a, cudaMemcpyAsync(v, a->diag_out, sizeof v, cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
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

int shz_amr_leaves(shz_amr* a, int32_t* n, int32_t* slots, int32_t* levels, int32_t* coords) {
  if (!a || !n) return SHZ_E_CONFIG;
  *n = n_leaves(a);
  for (int i = 0; i < n_leaves(a); i++) {
    const int s = a->h_leaves[i];
    const int32_t* row = a->h_bt.data() + (size_t)s * shz::amr::BT_STRIDE;
    if (slots) slots[i] = s;
    if (levels) levels[i] = row[0];
    if (coords)
      for (int ax = 0; ax < 3; ax++) coords[3 * i + ax] = row[1 + ax];
  }
  return 0;
}

int shz_amr_table(shz_amr* a, int32_t* out) {
  if (!a || !out) return SHZ_E_CONFIG;
  Dev dv(a->device);
  AMR_CUDA(a, cudaMemcpyAsync(out, a->d_bt, sizeof(int32_t) * a->cfg.cap * shz::amr::BT_STRIDE, cudaMemcpyDeviceToHost,
                              a->stream));
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  return 0;
}

int shz_amr_get_leaves_state(shz_amr* a, float* u1, float* u2) {
  if (!a || !u1 || !u2) return SHZ_E_CONFIG;
  Dev dv(a->device);
  const size_t bytes = (size_t)a->CB * sizeof(float4);
  for (int i = 0; i < n_leaves(a); i++) {
    const size_t s = (size_t)a->h_leaves[i] * a->CB;
    AMR_CUDA(a, cudaMemcpyAsync(u1 + (size_t)i * a->CB * 4, a->u1[a->cur] + s, bytes, cudaMemcpyDeviceToHost, a->stream));
    AMR_CUDA(a, cudaMemcpyAsync(u2 + (size_t)i * a->CB * 4, a->u2[a->cur] + s, bytes, cudaMemcpyDeviceToHost, a->stream));
  }
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  return 0;
}

int shz_amr_flags(shz_amr* a, float* out) {
  if (!a || !out) return SHZ_E_CONFIG;
  const size_t n = std::min<size_t>(a->h_flags.size(), (size_t)a->cfg.cap);
  std::memset(out, 0, sizeof(float) * a->cfg.cap);
  std::memcpy(out, a->h_flags.data(), n * sizeof(float));
  return 0;
}

int shz_amr_prims(shz_amr* a, int32_t slot, float* w1, float* w2) {
  if (!a || !w1 || !w2 || slot < 0 || slot >= a->cfg.cap) return SHZ_E_CONFIG;
  Dev dv(a->device);
  const size_t n = (size_t)a->WN, o = (size_t)slot * n;
  AMR_CUDA(a, cudaMemcpyAsync(w1, a->L.w1 + o, n * sizeof(float4), cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaMemcpyAsync(w2, a->L.w2 + o, n * sizeof(float4), cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  return 0;
}

int shz_amr_regrid_table(shz_amr* a, int32_t* out) {
  if (!a || !out) return SHZ_E_CONFIG;
  const size_t n = (size_t)a->cfg.cap * shz::amr::RG_STRIDE;
  std::memset(out, 0, n * sizeof(int32_t));
  std::memcpy(out, a->h_rg.data(), std::min(n, a->h_rg.size()) * sizeof(int32_t));
  return 0;
}

int shz_amr_ghost_map(shz_amr* a, int32_t slot, int32_t* out) {
  if (!a || !out || slot < 0 || slot >= a->cfg.cap) return SHZ_E_CONFIG;
  Dev dv(a->device);
  AMR_CUDA(a, shz::amr_launch_ghost_map(a->L, slot, a->d_ghost, a->stream));
  AMR_CUDA(a, cudaMemcpyAsync(out, a->d_ghost, sizeof(int32_t) * a->WN * 5, cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  return 0;
}

int shz_amr_profile(shz_amr* a, int32_t n, shz_profile_result* out) {
  if (!a || !out || n < 1) return SHZ_E_CONFIG;
  Dev dv(a->device);
  cudaEvent_t e0, e1;
  AMR_CUDA(a, cudaEventCreate(&e0));
  AMR_CUDA(a, cudaEventCreate(&e1));
  const long long l0 = a->launches;
  AMR_CUDA(a, cudaEventRecord(e0, a->stream));
  int taken = 0;
  int rc = step_n(a, n, &taken);
  AMR_CUDA(a, cudaEventRecord(e1, a->stream));
  AMR_CUDA(a, cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if ((rc = check_err(a))) return rc;
  out->steps = taken;
  out->total_ms = ms;
  out->sweep_ms = ms;
  out->launches = a->launches - l0;
  return 0;
}

int64_t shz_amr_kernel_launches(const shz_amr* a) { return a ? a->launches : 0; }

int shz_amr_bins(shz_amr* a, int32_t* bins, float* rates) {
  if (!a || !bins) return SHZ_E_CONFIG;
  Dev dv(a->device);
  const int cap = a->cfg.cap;
  if (a->cfg.time_bins <= 0) {
    std::memset(bins, 0, (size_t)(cap + 1) * sizeof(int32_t));
    if (rates) std::memset(rates, 0, (size_t)cap * sizeof(float));
    return 0;
  }
  AMR_CUDA(a, cudaMemcpyAsync(bins, a->d_bins[0], (size_t)(cap + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, a->stream));
  if (rates) AMR_CUDA(a, cudaMemcpyAsync(rates, a->d_brate, (size_t)cap * sizeof(float), cudaMemcpyDeviceToHost, a->stream));
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  return check_err(a);
}

int shz_amr_bin_work(shz_amr* a, int64_t* cycles, int64_t* updates, int64_t* single, int32_t* paused) {
  if (!a) return SHZ_E_CONFIG;
  if (cycles) *cycles = a->bin_cycles;
  if (updates) *updates = a->bin_updates;
  if (single) *single = a->bin_single;
  if (paused) *paused = a->bin_pause;
  return 0;
}

int shz_amr_reset_mesh(shz_amr* a, const shz_mesh_spec* m) {
  if (!a || !m || m->n < 1 || !m->levels || !m->coords) return SHZ_E_CONFIG;
  int root[3];
  for (int ax = 0; ax < 3; ax++) {
    if (m->block_size[ax] < 1 || m->root_size[ax] < m->block_size[ax] || m->root_size[ax] % m->block_size[ax] ||
        !(m->hi[ax] > m->lo[ax]))
      return fail(a, SHZ_E_CONFIG, "the snapshot's root grid along axis %d is not whole blocks over a box", ax);
    root[ax] = m->root_size[ax] / m->block_size[ax];
  }
  Dev dv(a->device);
  const shz_amr_config& c = a->cfg;
  // The snapshot's leaves by level and position (SnapshotSampler, io/snapshot.ts): 20 bits per
  // axis and the level above them.
  auto key = [](int l, long long i, long long j, long long k) {
    return ((uint64_t)l << 60) | ((uint64_t)k << 40) | ((uint64_t)j << 20) | (uint64_t)i;
  };
  std::unordered_map<uint64_t, int> index;
  index.reserve((size_t)m->n * 2);
  int top = 0;
  for (int b = 0; b < m->n; b++) {
    const int l = m->levels[b];
    if (l < 0 || l > 15) return fail(a, SHZ_E_CONFIG, "snapshot block %d: level %d", b, l);
    for (int ax = 0; ax < 3; ax++) {
      const long long span = (long long)root[ax] << l;
      if (m->coords[3 * b + ax] < 0 || m->coords[3 * b + ax] >= span || span > (1 << 20))
        return fail(a, SHZ_E_CONFIG, "snapshot block %d lies outside its root grid", b);
    }
    index.emplace(key(l, m->coords[3 * b], m->coords[3 * b + 1], m->coords[3 * b + 2]), b);
    top = std::max(top, l);
  }
  // SnapshotSampler.level at a point: the finest leaf whose block holds it; -1 if none does.
  auto level_at = [&](const double x[3]) {
    double f[3];
    for (int ax = 0; ax < 3; ax++) {
      const double v = (x[ax] - m->lo[ax]) / (m->hi[ax] - m->lo[ax]);
      // an axis of one cell is the same at every point along it
      f[ax] = m->root_size[ax] == 1 ? 0.0 : std::min(std::max(v, 0.0), 1 - 1e-7);
    }
    for (int l = top; l >= 0; l--) {
      long long at[3];
      for (int ax = 0; ax < 3; ax++) {
        const long long span = (long long)root[ax] << l;
        at[ax] = std::min((long long)std::floor(f[ax] * (double)span), span - 1);
      }
      if (index.count(key(l, at[0], at[1], at[2]))) return l;
    }
    return -1;
  };
  try {
    a->tree.reset(new BlockTree(c.ndim, c.nr, c.max_level, c.cap, c.hydro.bc_lo, c.hydro.bc_hi));
  } catch (const std::exception& e) {
    return fail(a, SHZ_E_CONFIG, "%s", e.what());
  }
  const double dx0 = dx0_of(c), half = c.box / 2;
  const bool three = c.ndim == 3;
  bool uncovered = false;
  // finerInSnapshot (amr_sim.ts:1867-1875): the snapshot is finer than the block at the centre of
  // one of its children; levels shifted to this run's root and never below 0.
  auto finer = [&](const shz::amr::Block* b) {
    const double size = shz::amr::BS * dx0 / (double)(1 << b->level);
    for (int o = 0; o < (three ? 8 : 4); o++) {
      double x[3] = {0, 0, 0};
      for (int ax = 0; ax < (three ? 3 : 2); ax++) x[ax] = (b->c[ax] + (((o >> ax) & 1) + 0.5) / 2) * size - half;
      const int l = level_at(x);
      if (l < 0) {
        uncovered = true;
        return 0.0;
      }
      if (std::max(0, l + m->shift) > b->level) return 1.0;
    }
    return 0.0;
  };
  for (int pass = 0; pass < c.max_level; pass++) {
    std::vector<RegridOp> ops;
    try {
      ops = a->tree->adapt(finer, 0.5, -1.0);
    } catch (const std::exception& e) {
      return fail(a, SHZ_E_CONFIG, "adapt: %s", e.what());
    }
    if (uncovered) return fail(a, SHZ_E_CONFIG, "the snapshot does not cover the whole domain");
    if (ops.empty()) break;
  }
  int rc = upload_tables(a);
  if (rc) return rc;
  a->cur = 0;
  a->slot = 0;
  const size_t bytes = (size_t)c.cap * a->CB * sizeof(float4);
  AMR_CUDA(a, cudaMemsetAsync(a->u1[0], 0, bytes, a->stream));
  AMR_CUDA(a, cudaMemsetAsync(a->u2[0], 0, bytes, a->stream));
  a->since_check = 0;
  a->flags_due = false;
  reset_bins(a);
  return write_clock(a, 0.0, 0);
}

int shz_amr_set_leaves_state(shz_amr* a, const float* u1, const float* u2) {
  if (!a || !u1 || !u2) return SHZ_E_CONFIG;
  Dev dv(a->device);
  const size_t bytes = (size_t)a->CB * sizeof(float4);
  for (int i = 0; i < n_leaves(a); i++) {
    const size_t s = (size_t)a->h_leaves[i] * a->CB;
    AMR_CUDA(a, cudaMemcpyAsync(a->u1[a->cur] + s, u1 + (size_t)i * a->CB * 4, bytes, cudaMemcpyHostToDevice, a->stream));
    AMR_CUDA(a, cudaMemcpyAsync(a->u2[a->cur] + s, u2 + (size_t)i * a->CB * 4, bytes, cudaMemcpyHostToDevice, a->stream));
  }
  AMR_CUDA(a, cudaStreamSynchronize(a->stream));
  return 0;
}

int shz_amr_set_clock(shz_amr* a, double t, int64_t steps) {
  if (!a || !std::isfinite(t) || steps < 0) return SHZ_E_CONFIG;
  Dev dv(a->device);
  reset_bins(a);
  return write_clock(a, t, steps);
}

}  // extern "C"
