/*
 * shaderous_b200 — C ABI of a B200-native compressible-hydro step.
 *
 * This is the drop-in boundary for the reference's simulation driver. In the reference
 * (guillochon/shaderous), TypeScript callers hold a `Simulation` (src/sim.ts:465-628) created by
 * `createSim` (src/create.ts:58-61) and drive it with `run({steps, until, timeoutMs})`
 * (src/ui/api.ts:188-210, 538). The functions below are what a Node N-API addon binds in its
 * place; every one is plain C: POD structs, host pointers and sizes, an int status.
 *
 * Conventions
 *  - Every function returns 0 on success or a negative SHZ_E* code; shz_last_error() gives the
 *    message of the last failure on a handle (UTF-8, owned by the handle).
 *  - Host buffers belong to the caller; device memory belongs to the handle. No device pointer
 *    escapes except through shz_state_device() and the slab functions below, documented there.
 *  - A handle is not re-entrant: callers serialise calls on one handle, as the reference's API
 *    serialises every call (src/ui/api.ts:1414-1416). Different handles may be used from
 *    different threads; each owns one CUDA stream.
 *  - State layout: two float4 arrays per cell, x fastest then y then z, as the reference's
 *    readState() returns them (src/sim.ts:3790-3808):
 *      u1 = (rho, rho vx, rho vy, rho vz), u2 = (E, e_int, rho s, solid flag = 0).
 */
#ifndef SHADEROUS_B200_H
#define SHADEROUS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define SHZ_OK 0
#define SHZ_E_CONFIG (-1)    /* a configuration or argument the library refuses */
#define SHZ_E_OOM (-2)       /* device memory could not be allocated */
#define SHZ_E_NAN (-3)       /* the clock became NaN (src/sim.ts:3708; api.ts settle) */
#define SHZ_E_CUDA (-4)      /* a CUDA call failed; the message names it */
#define SHZ_E_TIMEOUT (-5)   /* a device-side bounded wait ran out */
#define SHZ_E_CANCELLED (-6) /* a request was cancelled */
#define SHZ_E_NODEV (-7)     /* no usable sm_100 device */

/* Boundary codes, as src/problems/boundaries.ts:20-24 and src/reference/hydro.ts:216-220. */
#define SHZ_BC_PERIODIC 0
#define SHZ_BC_OUTFLOW 1
#define SHZ_BC_REFLECT 2
/* z faces only: one slab of a grid split along z over several handles (one per GPU). The handle
 * stores the face's ghost planes (shz_halo_depth) beyond the slab; the caller fills them with the
 * neighbouring slab's planes before every step (shz_halo_device). No counterpart in the reference,
 * which runs one grid on one GPU (docs/architecture.md:695-700). */
#define SHZ_BC_HALO 3

/* Reconstructions: the reference's limiters (src/reference/hydro.ts:30-46) plus PPM. */
#define SHZ_RECON_MINMOD 0
#define SHZ_RECON_MC 1
#define SHZ_RECON_VANLEER 2
#define SHZ_RECON_KOREN 3
#define SHZ_RECON_PPM 4 /* Colella & Woodward 1984 edge values; no counterpart in the reference */

#define SHZ_RIEMANN_HLLC 0
#define SHZ_RIEMANN_HLL 1

/*
 * Run configuration: the hot-path subset of the reference's SimConfig (src/sim.ts:48-265),
 * with the reference's defaults from configFor (src/sim.ts:645-742) set by shz_config_default().
 */
typedef struct shz_config {
  int32_t n[3];         /* cells along x, y, z; 1 along a collapsed axis (1D: ny = nz = 1; 2D: nz = 1) */
  double dx;            /* cell size (the reference's box / n) */
  double gamma;         /* ideal-gas adiabatic index (src/eos/ideal.wgsl) */
  int32_t bc_lo[3];     /* SHZ_BC_* per axis, lower face */
  int32_t bc_hi[3];     /* SHZ_BC_* per axis, upper face */
  double cfl;           /* Courant number (default 0.8) */
  double rho_floor;     /* default 1e-10 */
  double p_floor;       /* default 1e-14 */
  double eta_dual;      /* dual-energy switch (default 1e-3) */
  double shock_thresh;  /* shock flag's relative pressure jump (default 0.5) */
  int32_t riemann;      /* SHZ_RIEMANN_* (default HLLC) */
  int32_t recon;        /* SHZ_RECON_* (default KOREN) */
  int32_t isentropic;   /* density along the adiabat (default 1; ignored with PPM) */
  int32_t signal_dims;  /* multiple of c in the signal rate: 3 as src/reference/hydro.ts:254 (default) */
  double t_end;         /* the clock stops here (default +inf) */
  double dt_max;        /* largest step (default +inf) */
  int32_t device;       /* CUDA device ordinal the handle lives on (default 0) */
} shz_config;

/* run() options and result, as RunOptions / RunResult (src/ui/api.ts:188-210). */
typedef struct shz_run_opts {
  int64_t steps;      /* take at most this many steps; < 0 for no limit */
  double until;       /* run until the clock reads this time; NaN for none */
  double timeout_ms;  /* give up after this much wall time; <= 0 for none */
} shz_run_opts;

#define SHZ_STOP_STEPS 0
#define SHZ_STOP_TIME 1
#define SHZ_STOP_END 2
#define SHZ_STOP_TIMEOUT 3

typedef struct shz_run_result {
  double t;        /* clock after the call */
  double dt;       /* step the clock would take next (0 when held at a stop) */
  int64_t steps;   /* steps taken since the last reset */
  int64_t taken;   /* steps taken by this call */
  double seconds;  /* wall time of the call */
  int32_t stopped; /* SHZ_STOP_* */
  double last_dt;  /* length of the last step taken */
} shz_run_result;

/* Conservation totals in float64 (compensated sums), as the reference's Diagnostics
 * (src/sim.ts:1810-1862, channels of src/hydro/diagnostics.wgsl). dV = dx^ndim. */
typedef struct shz_diag {
  double t, dt;
  int64_t steps;
  double mass;         /* sum rho dV */
  double momentum[3];  /* sum rho v dV */
  double e_kin;        /* sum 1/2 rho v^2 dV */
  double e_int;        /* sum (E - 1/2 rho v^2) dV */
  double e_tot;        /* sum E dV */
  double max_mach;     /* max |v| / c */
  double floored;      /* cells at the density or pressure floor */
} shz_diag;

/* Built-in problems, initialised on the host in float64 at cell centres (box centred on 0, as
 * src/reference/hydro.ts:200 and src/domain.ts:15) and rounded once to float32. */
#define SHZ_PROB_SOD 0       /* shock tube along `axis`: left (a[0..2] = rho,u,p) for x<0, right (a[3..5]); s = 1 on the left */
#define SHZ_PROB_KH 1        /* Kelvin-Helmholtz slab: rho_in a[0], rho_out a[1], v a[2], p a[3], kick a[4], noise sigma a[5] */
#define SHZ_PROB_TGV 2       /* Taylor-Green vortex on [0, 2 pi]^3: rho a[0], p0 a[1], amplitude a[2] */
#define SHZ_PROB_SEDOV 3     /* point blast: rho a[0], p a[1], energy a[2], radius in cells a[3] */
#define SHZ_PROB_ADVECT 4    /* smooth density wave: rho = a[0] + a[1] sin(2 pi x / L), v = (a[2], a[3], a[4]), p = a[5] */
#define SHZ_PROB_BLAST 5     /* pressure sphere: rho_in a[0], p_in a[1], rho_out a[2], p_out a[3], radius (box units) a[4] */
#define SHZ_PROB_GAUSS 6     /* gaussian pulse in 3D: rho = a[0] + exp(-r2/a[1]), v = (a[2],a[3],a[4]) , p = a[5] + 0.5 exp(-r2/a[6]) */

/* The rest of the reference's Diagnostics channels (hydro/diagnostics.wgsl channels 6, 9-23;
 * src/sim.ts:1808-1862): the totals above, the [min, max] over the cells of density,
 * temperature ((gamma - 1) e_int / rho), scalar (rho s / rho), pressure and speed (`ranges`, in
 * the reference's FIELDS order), and the centre of mass from the box centre (`com`). The
 * gravitational, Jeans and burning channels are zero: no gravity or burning on this path. */
typedef struct shz_diag_ext {
  shz_diag base;
  double range[5][2];
  double com[3];
  double e_grav;
  double jeans_unresolved;
  double nuclear_heating;
} shz_diag_ext;

typedef struct shz_problem {
  int32_t kind;    /* SHZ_PROB_* */
  int32_t axis;    /* SOD: normal axis */
  uint64_t seed;   /* KH noise */
  double a[8];     /* parameters, per kind above */
} shz_problem;

typedef struct shz_sim shz_sim;

/* Fill `cfg` with the reference's defaults for an n[0] x n[1] x n[2] grid of cell size dx. */
int shz_config_default(shz_config* cfg, int32_t nx, int32_t ny, int32_t nz, double dx);

/* Replaces createSim / Sim.create (src/create.ts:58-61, src/sim.ts:2283): validates the
 * configuration, allocates the device state and builds the step. */
int shz_create(const shz_config* cfg, shz_sim** out);

/* Replaces Simulation.destroy (src/sim.ts:465-628). */
void shz_destroy(shz_sim* sim);

/* Message of the last failure on `sim` (or of the last shz_create failure when sim is NULL). */
const char* shz_last_error(const shz_sim* sim);

/* Replaces Sim.reset with a built-in problem (src/sim.ts:2704-2848): the clock goes to 0. */
int shz_reset_problem(shz_sim* sim, const shz_problem* prob);

/* Host float64 primitives (rho, vx, vy, vz, p, s per cell, x fastest) of planes k0..k1-1 of a
 * problem on the grid of `cfg`: the same numbers shz_reset_problem() rounds to float32. */
int shz_problem_prims(const shz_config* cfg, const shz_problem* prob, int32_t k0, int32_t k1, double* prims);

/* Replaces Simulation.setState (src/sim.ts:3031): host float32 state, `ncell` cells, layout above.
 * Keeps the clock. */
int shz_set_state(shz_sim* sim, const float* u1, const float* u2, size_t ncell);

/* Replaces Simulation.readState (src/sim.ts:3790-3808): copies the state into host buffers. */
int shz_get_state(shz_sim* sim, float* u1, float* u2, size_t ncell);

/* Replaces encodeSteps + submit (src/sim.ts:3187-3328): enqueue `n` steps; returns at once.
 * Steps past t_end hold the clock (dt = 0) and leave the state as it is. */
int shz_step(shz_sim* sim, int32_t n);

/* Replaces run() (src/ui/api.ts:538): steps until `steps`, `until` or the timeout, whichever
 * comes first; the step that reaches `until` is shortened to land on it. Blocking. */
int shz_run(shz_sim* sim, const shz_run_opts* opts, shz_run_result* res);

/* Replaces readDiagnostics (src/sim.ts:3602-3650). Blocking. */
int shz_diagnostics(shz_sim* sim, shz_diag* out);

/* The device clock (src/hydro/common.wgsl Clock): t, the next dt and the steps taken. Blocking. */
int shz_clock(shz_sim* sim, double* t, double* dt, int64_t* steps);

/* Set the clock (a restart, RestartState src/sim.ts:1865). */
int shz_set_clock(shz_sim* sim, double t, int64_t steps);

/* Change the stop time t_end (the reference's writeParams with cfg.tEnd). */
int shz_set_t_end(shz_sim* sim, double t_end);

/* Wait for the handle's queued work. */
int shz_sync(shz_sim* sim);

/* Totals and the extended channels (shz_diag_ext), as Simulation.diagnostics() returns them. */
int shz_diagnostics_ext(shz_sim* sim, shz_diag_ext* out);

/* Device pointers of the current state (two float4 arrays, layout above), valid until the next
 * step or destroy; for callers that keep data on the device (benchmarks, interop). */
int shz_state_device(shz_sim* sim, void** u1, void** u2);

/*
 * A grid split into z-slabs, one handle per GPU (SHZ_BC_HALO faces). Before every step the
 * caller, on the handle's stream:
 *   1. copies each halo face's `inner` planes into the neighbouring slab's `ghost` planes of the
 *      facing side (and receives its own ghosts likewise): NCCL send/recv between GPUs;
 *   2. replaces the rate word with its maximum over all slabs (an all-reduce of uint32 max: the
 *      word holds a non-negative float's bits), so that every slab takes the same dt;
 * then calls shz_step(sim, 1). The pointers change parity every step: query them each time.
 * No counterpart in the reference (single GPU).
 */
/* Load planes k0 .. k0 + nz - 1 of a built-in problem sampled on the whole grid `grid` (nx, ny
 * and dx as the slab's) into the slab; the clock goes to 0. */
int shz_reset_problem_slab(shz_sim* sim, const shz_config* grid, const shz_problem* prob, int32_t k0);
/* Stored ghost planes of a halo face: 3 with PPM, else 2. */
int shz_halo_depth(const shz_sim* sim, int32_t* planes);
/* Face `side` (0 lower z, 1 upper z) of the current state: its inner planes (the slab's own
 * planes next to the face) and its ghost planes (stored beyond it), each `bytes` long in u1 and
 * in u2 (depth x nx x ny float4, x fastest). */
int shz_halo_device(shz_sim* sim, int32_t side, void** inner_u1, void** inner_u2, void** ghost_u1, void** ghost_u2,
                    size_t* bytes);
/* The device word the next step's clock reads its rate from (uint32 bits of the largest
 * rate / dx over this slab after its last step, or after shz_set_state / shz_reset_problem). */
int shz_rate_device(shz_sim* sim, void** rate);
/* The handle's CUDA stream (a cudaStream_t), to order the caller's transfers with the steps. */
int shz_stream(shz_sim* sim, void** stream);

/* Per-pass timing of `n` steps with CUDA events on the handle's stream, as the reference's
 * Sim.profile(reps) (src/sim.ts:3541) and its per-pass timestamps (src/gpu/timing.ts:232):
 * total device time of the steps, and the summed time of the sweep kernels alone. Blocking. */
typedef struct shz_profile_result {
  int32_t steps;
  double total_ms;   /* first clock kernel's start to last sweep's end */
  double sweep_ms;   /* sum over the n sweeps of each sweep's own duration */
  int64_t launches;  /* kernels launched for the n steps */
} shz_profile_result;
int shz_profile(shz_sim* sim, int32_t n, shz_profile_result* out);

/*
 * The adaptive grid's block tree (host), deciding slot for slot as the reference's BlockTree
 * (src/amr/tree.ts:106-824), and its flat tables for bit-exact checks. Blocks hold 16^ndim cells
 * (BS, tree.ts:14); the block table has 32 ints per slot (BT_STRIDE, layout tree.ts:42-60), the
 * regrid table 12 (RG_STRIDE, tree.ts:62-66).
 */
#define SHZ_AMR_BS 16
#define SHZ_AMR_BT_STRIDE 32
#define SHZ_AMR_RG_STRIDE 12
typedef struct shz_tree shz_tree;
/* new BlockTree(ndim, nr, maxLevel, cap, bcLo, bcHi, edgeBalance) (tree.ts:139). */
int shz_tree_create(int32_t ndim, int32_t nr, int32_t max_level, int32_t cap, const int32_t bc_lo[3],
                    const int32_t bc_hi[3], int32_t edge_balance, shz_tree** out);
void shz_tree_destroy(shz_tree* t);
const char* shz_tree_error(void);
/* adapt((b) => indicator[b.slot], hi, lo) (tree.ts:489). regrid: cap * 12 ints or NULL;
 * changed: 0 if the tree did not change (adapt returned null). */
int shz_tree_adapt(shz_tree* t, const double* indicator_by_slot, double hi, double lo, int32_t* regrid, int32_t* changed);
/* The steps the last adapt took, flattened [what, level, c0..c(ndim-1)] per step (tree.ts:574). */
int shz_tree_last_steps(const shz_tree* t, int32_t* out, int32_t max_ints, int32_t* n_ints);
/* replayAdapt(steps) (tree.ts:579): the same flattened form. */
int shz_tree_replay(shz_tree* t, const int32_t* steps, int32_t n_ints, int32_t* regrid, int32_t* changed);
/* refine(get(level, c)) (tree.ts:366): *n_split = blocks split (0 if refused). */
int shz_tree_refine(shz_tree* t, int32_t level, const int32_t c[3], int32_t* n_split);
/* neighbor(get(level, c), f) (tree.ts:283): kind 0 same, 1 coarse, 2 boundary; slot or type. */
int shz_tree_neighbor(const shz_tree* t, int32_t level, const int32_t c[3], int32_t f, int32_t* kind, int32_t* slot_or_type);
int shz_tree_table(const shz_tree* t, int32_t* out);                  /* cap * 32 ints */
/* lists() (tree.ts:695): every block coarsest first, the leaves, blocks per level. */
int shz_tree_lists(const shz_tree* t, int32_t* all, int32_t* leaves, int32_t* per_level, int32_t* n_all, int32_t* n_leaves);
int64_t shz_tree_index_grid_size(const shz_tree* t);
int shz_tree_index_grid(const shz_tree* t, uint32_t* out);             /* leaf slot per finest block cell */
/* count, free slots, leaves, deepest level, highest slot used */
/* indexGrid(boxes) (tree.ts:721-803): the index grid (as shz_tree_index_grid) and the boxes that
 * changed since the last call of this function, 6 ints each (origin x, y, z, size x, y, z): the
 * whole grid on the first call, else runs of changed rows; a copy updated only inside them stays
 * equal to the grid. *n_boxes = the boxes found (at most max_boxes are written). */
int shz_tree_index_grid_boxes(shz_tree* t, uint32_t* out, int32_t* boxes, int32_t max_boxes, int32_t* n_boxes);
/* The bcLo / bcHi setters (tree.ts:193-199): boundary types of a built tree; tables read after it
 * show them. */
int shz_tree_set_bc(shz_tree* t, const int32_t bc_lo[3], const int32_t bc_hi[3]);
int shz_tree_stats(const shz_tree* t, int32_t* blocks, int32_t* free_slots, int32_t* leaves, int32_t* deepest, int32_t* high_slot);

/*
 * A run on the adaptive block grid: replaces AmrSim (src/amr/amr_sim.ts:178) behind the same
 * Simulation interface. The domain is a cube of side `box` (centred on 0) covered by nr^ndim
 * root blocks of 16^ndim cells, refined up to max_level levels in a budget of `cap` block slots.
 * A step is assemble -> clock -> predict -> update (src/amr/amr_sim.ts:2709-2946), captured as
 * one CUDA graph; every regrid_every steps (REGRID_EVERY = 8, amr_sim.ts:73) the Löhner
 * indicator (amr/flag.wgsl) drives BlockTree.adapt and the new leaves are filled
 * (amr/regrid.wgsl). The check is made at the start of the next step, from that step's own
 * assemble, as the reference applies a re-mesh at the start of the next steps (applyRegrid).
 * Limiters minmod, mc, vanleer and koren (PPM needs a third ghost layer).
 */
typedef struct shz_amr_config {
  shz_config hydro;     /* physics and boundaries; n[] and dx are ignored */
  int32_t ndim;         /* 2 or 3 */
  int32_t nr;           /* root blocks per side */
  int32_t max_level;    /* deepest level (0..7) */
  int32_t cap;          /* block slots (leaves and parents) */
  double box;           /* side of the domain; level-0 cell size box / (16 nr) */
  double refine_hi;     /* refine leaves whose indicator exceeds this */
  double refine_lo;     /* merge siblings whose indicators are all below this */
  int32_t regrid_every; /* steps between refinement checks (0: never) */
  int32_t two_pass;     /* 0: one fused sweep per leaf (predict, fluxes and update from the
                           primitives); 1: the reference's two passes, predict into a half-step
                           atlas then update (amr_sim.ts:2709-2946), which costs that atlas's
                           memory; both give the same state to rounding */
  int32_t time_bins;    /* per-block timesteps (SimConfig.timeBins, amr_sim.ts:1002-1010): 0 off,
                           else up to 5 bins, time advancing in cycles of 2^time_bins substeps of
                           the fastest block's step (amr/bins_*.wgsl); run with the two-pass
                           kernels, which keep each block's half step for its slower neighbours */
  int32_t time_bins_always; /* 1: never pause the cycles when they save too little
                               (SimConfig.timeBinsAlways, amr_sim.ts:2992-3020) */
} shz_amr_config;
typedef struct shz_amr shz_amr;

int shz_amr_create(const shz_amr_config* cfg, shz_amr** out);
void shz_amr_destroy(shz_amr* a);
const char* shz_amr_error(const shz_amr* a);
/* Initial conditions of a built-in problem on the adaptive grid: the mesh is built by up to
 * max_level passes of adapt() over the sampled state (amr_sim.ts:1924-2100), each leaf sampled at
 * its own cell centres; blocks that a problem's discontinuity crosses count as flagged. */
int shz_amr_reset_problem(shz_amr* a, const shz_problem* prob);
int shz_amr_step(shz_amr* a, int32_t n);
int shz_amr_run(shz_amr* a, const shz_run_opts* opts, shz_run_result* res);
int shz_amr_diagnostics(shz_amr* a, shz_diag* out);
int shz_amr_clock(shz_amr* a, double* t, double* dt, int64_t* steps);
/* Totals and the extended channels over the leaves (shz_diag_ext). */
int shz_amr_diagnostics_ext(shz_amr* a, shz_diag_ext* out);
/* Run the refinement check now (flag, adapt, regrid); *changed = 1 if the mesh changed. */
int shz_amr_regrid(shz_amr* a, int32_t* changed);
/* The leaves, coarsest first (lists().leaves): slots, levels and block coordinates (3 per leaf). */
int shz_amr_leaves(shz_amr* a, int32_t* n_leaves, int32_t* slots, int32_t* levels, int32_t* coords);
/* The block table on the device (cap * 32 ints), read back: the tree's, plus two words the passes
 * use: 26 the block's grid (0 here) and 27 a leaf's first entry in the fine-flux buffer of its
 * faces matched to refined neighbours (-1 for none). */
int shz_amr_table(shz_amr* a, int32_t* out);
/* State of the leaves in lists().leaves order: 16^ndim cells each, x fastest, float4 u1 and u2. */
int shz_amr_get_leaves_state(shz_amr* a, float* u1, float* u2);
/* The last refinement indicators per slot (cap floats). */
int shz_amr_flags(shz_amr* a, float* out);
/* The primitive region of block `slot` as the last assemble left it (a step's first pass, or a
 * refinement check's): 20^ndim texels, x fastest, w1 = (rho, vx, vy, vz) and w2 = (p, s, cs, 0)
 * as float4 each (AmrSim's W1/W2 atlas texels, amr/assemble.wgsl:78-154; this build keeps the
 * sound speed where the reference keeps the internal energy). For checks against an oracle. */
int shz_amr_prims(shz_amr* a, int32_t slot, float* w1, float* w2);
/* The regrid table of the last re-mesh (cap * 12 ints, BlockTree.regridTable,
 * src/amr/tree.ts:681-693: kind 1 copy / 2 prolong / 3 restrict, source slot, octant, children);
 * zero before the first. */
int shz_amr_regrid_table(shz_amr* a, int32_t* out);
/* The device's ghost classification of block `slot`: (kind, source slot, l0, l1, l2) for each of
 * the 20^ndim texels of its primitive region, x fastest (amr/grid.wgsl ghost_src). */
int shz_amr_ghost_map(shz_amr* a, int32_t slot, int32_t* out);
int shz_amr_profile(shz_amr* a, int32_t n, shz_profile_result* out);
int64_t shz_amr_kernel_launches(const shz_amr* a);
/* Per-block timesteps. The bin table of the last cycle (AmrSim.readBins, amr_sim.ts:4283): cap + 1
 * ints, [0] the substep last taken, [1 + slot] the block's bin; and, if rates is not null, the
 * blocks' own signal rates per unit cell size that the cycle's bins were formed from (cap floats,
 * leaves only). Both are zero before the first cycle. */
int shz_amr_bins(shz_amr* a, int32_t* bins, float* rates);
/* The work of the cycles so far (AmrSim.binWork, amr_sim.ts:1663): cycles taken, block updates
 * made (deposits included) and the updates single steps would have made; *paused: single steps
 * left before the cycles resume (the start of a run, or a pause when they saved too little). */
int shz_amr_bin_work(shz_amr* a, int64_t* cycles, int64_t* updates, int64_t* single, int32_t* paused);

/* Restart on blocks from a snapshot (io/capture.ts restartFrom, amr_sim.ts:1867-1875 and
 * 1943-1971). The snapshot's leaves: n blocks, each a level and a position in blocks at that level
 * (3 ints, z 0 in 2D), on a root grid of root_size[3] cells in blocks of block_size[3] cells,
 * spanning [lo, hi] along each axis (the Snapshot's rootSize, blockSize, lo, hi); shift is how
 * many levels finer the file's root cells are than this run's (levels count from the file's
 * root). */
typedef struct {
  int32_t n;
  const int32_t* levels;
  const int32_t* coords;
  int32_t root_size[3];
  int32_t block_size[3];
  double lo[3], hi[3];
  int32_t shift;
} shz_mesh_spec;
/* Rebuild the tree as a restart does: up to max_level passes of adapt() that refine every leaf
 * the snapshot is finer than at one of its children's centres and merge none. The leaves' state
 * is zero afterwards (set it with shz_amr_set_leaves_state) and the clock at 0. A point the
 * snapshot's leaves do not cover is refused. */
int shz_amr_reset_mesh(shz_amr* a, const shz_mesh_spec* mesh);
/* Replace the state of every leaf, leaves in shz_amr_leaves order, each as shz_amr_get_leaves_state
 * gives it (16^ndim cells, x fastest, float4 u1 and u2). */
int shz_amr_set_leaves_state(shz_amr* a, const float* u1, const float* u2);
/* Set the clock's time and step count (a restart's, Restart.time and .steps). */
int shz_amr_set_clock(shz_amr* a, double t, int64_t steps);

/*
 * Serving: independent hydro runs ("requests") of uneven sizes kept resident in HBM and advanced
 * together. Every request is a uniform grid of 16^ndim-cell blocks; the blocks of all running
 * requests form one work list that the adaptive grid's passes walk each step (one CUDA graph per
 * step, per-request parameters and clocks). Requests are admitted against a memory budget as
 * block slots free up, between rounds of `round_steps` steps (continuous batching). No
 * counterpart in the reference, whose nearest form is its sequential `sweep` runs
 * (tools/headless/cli.mjs:367-380).
 */
typedef struct shz_request {
  int32_t ndim;          /* 2 or 3 */
  int32_t n;             /* cells per side, a multiple of 16 */
  int32_t steps;         /* steps to take */
  int32_t bc;            /* boundary code on every face */
  double gamma;
  double arrival;        /* seconds after the stream starts (shz_server_run_stream) */
  shz_problem problem;   /* initial condition on the unit box */
} shz_request;

typedef struct shz_server_config {
  shz_config hydro;      /* scheme and floors for every request (gamma and bc come per request) */
  double budget_bytes;   /* device memory for resident request state */
  int32_t max_grids;     /* requests in flight at most */
  int32_t round_steps;   /* steps between admission and completion checks */
  int32_t keep_states;   /* 1: keep each finished request's state for shz_server_state */
  int32_t direct_large;  /* 1: a request of at least 2^18 cells (2D) or 2^21 (3D) runs as a uniform
                            grid (the fused sweep) on a stream of its own, its steps enqueued in the
                            same rounds as the batched blocks, within a quarter of the budget; 0:
                            every request on the block passes */
} shz_server_config;

typedef struct shz_server_stats {
  int64_t completed;
  double makespan_s;       /* first arrival to last completion */
  double p50_s, p99_s;     /* completion latency: finish - arrival */
  double mean_s;
  double zone_updates;     /* cells x steps over all requests */
  double zu_per_s;         /* zone_updates / makespan */
  int64_t max_concurrent;  /* requests in flight at once, at most */
  int64_t rounds;
  int64_t kernel_launches;
  double busy_s;           /* GPU-busy seconds (CUDA events): the batched server's rounds (per
                              round, the longer of its two engines' spans), or the plain loop's
                              runs; busy_s / makespan_s is the device's busy share */
} shz_server_stats;

typedef struct shz_server shz_server;
int shz_server_create(const shz_server_config* cfg, shz_server** out);
void shz_server_destroy(shz_server* s);
const char* shz_server_error(const shz_server* s);
/* Queue a request now; *id numbers it. */
int shz_server_submit(shz_server* s, const shz_request* req, int64_t* id);
/* Run rounds until every queued request has finished (or max_rounds rounds, if > 0). */
int shz_server_drain(shz_server* s, int32_t max_rounds);
/* Run a stream: request i is queued once the wall clock passes reqs[i].arrival seconds after the
 * call starts; returns when all are done, with latency statistics. */
int shz_server_run_stream(shz_server* s, const shz_request* reqs, int32_t n, shz_server_stats* out);
/* The conservation totals of a finished request, and (keep_states) its final state as uniform
 * arrays of n^ndim cells, x fastest. */
/* Cancel request `id` (called between other server calls, with no round in flight): a queued
 * request leaves the queue; a running one gives its block slots and clock back at once, and the
 * others go on as they would have. Its result and state then return SHZ_E_CANCELLED. Returns
 * SHZ_E_CONFIG for an unknown id or a request that has finished or was cancelled already. No
 * counterpart in the reference (whose runs stop by their RunOptions timeoutMs). */
int shz_server_cancel(shz_server* s, int64_t id);
/* The state of request `id` (called between other server calls): *status one of SHZ_REQ_*, and,
 * if steps_done is not null, the steps it has taken (its whole count once finished). No
 * counterpart in the reference (a page runs one simulation, whose clock run() reads back). */
#define SHZ_REQ_QUEUED 0
#define SHZ_REQ_RUNNING 1
#define SHZ_REQ_FINISHED 2
#define SHZ_REQ_CANCELLED 3
int shz_server_poll(shz_server* s, int64_t id, int32_t* status, int64_t* steps_done);
int shz_server_result(shz_server* s, int64_t id, shz_diag* diag);
int shz_server_state(shz_server* s, int64_t id, float* u1, float* u2);
/* The same stream run one request after another, each through the plain uniform-grid step
 * (shz_create / shz_reset_problem / shz_run / shz_destroy), for comparison. */
int shz_plain_run_stream(const shz_server_config* cfg, const shz_request* reqs, int32_t n, shz_server_stats* out);

/* Launches of the library's own kernels on this handle since creation. */
int64_t shz_kernel_launches(const shz_sim* sim);

/* Library version string. */
const char* shz_version(void);

/*
 * The launch-shape autotuner. No counterpart in the reference, whose WGSL passes have fixed
 * workgroup sizes chosen per kernel at build time (src/gpu/*.ts).
 *
 * The first time a handle runs a tunable kernel for a (kernel, ndim, reconstruction, isentropic,
 * size class) key, it times every candidate shape in place inside one real step, keeps the
 * fastest in a process-wide table, and uses it from then on (also in captured CUDA graphs).
 * Candidates differ only in launch shape, never in arithmetic: the state is the same whichever
 * wins. Kernels and their knobs:
 *   0 uniform sweep: tz = planes a CTA marches along z (3D); in 2D grids of at least 512 cells
 *     a side, the rows a CTA marches along y (smaller 2D grids take a tile form, 16 x 12 cells
 *     with a ring of halo cells, untuned; the two forms agree to rounding, each depth of one form
 *     gives the same bits);
 *   1 AMR assemble: variant = register budget (0: 1, 1: 2, 2: 3 CTAs per SM) of the one-pass
 *     kernel, or the split form (3: 2, 4: 3 CTAs per SM for its second pass): a light first
 *     pass for the blocks' own cells and same-level ghosts, then the ghosts beyond a level
 *     change over only the blocks that have them; 5, 6: the split form with its two passes side
 *     by side on a second stream; per_sm = CTAs of the work-list grid per SM;
 *   2 AMR fused sweep: per_sm;
 *   3 AMR fine-flux pass: per_sm;
 *   4 the per-block-timestep substeps' assemble: variant 1 one pass, 3 the split form (its
 *     second pass over every block of the substep's list); per_sm.
 */
typedef struct shz_tune_entry {
  int32_t kernel, ndim, recon, isentropic, size_class;  /* the key; size class = floor(log2 units) */
  int32_t variant, per_sm, tz;                          /* the choice (0: the kernel's default) */
  int32_t candidates;                                   /* shapes timed */
  float ms, default_ms;                                 /* mean time of the choice and of the default */
} shz_tune_entry;
/* Turn the tuner on (default) or off (every launch takes the default shape). Process-wide. */
int shz_tune_enable(int32_t on);
/* Pin one kernel's choice for every key, used instead of the tuned one; variant < 0 unpins.
 * Process-wide. AMR kernels (1-4 above): variant, per_sm with 0 for the default grid. The uniform
 * sweep (0): variant 0 and per_sm = its depth tz (0-1024; in 2D 0 is the tile form). */
int shz_tune_pin(int32_t kernel, int32_t variant, int32_t per_sm);
/* Forget every choice. */
void shz_tune_reset(void);

/* A check of the kernels' bounded waits on `device`: one CTA waits on an mbarrier phase that
 * nothing completes, with a short limit, and reports through its error word as a sweep whose bulk
 * copy never lands would (then the handle's calls return SHZ_E_TIMEOUT). *code is the kernel's
 * error code: 1 (the timeout) when the path works. No counterpart in the reference. */
int shz_selftest_wait_timeout(int32_t device, int32_t* code);
/* Copy up to `max` entries of the table; *n = entries in the table. */
int shz_tune_entries(shz_tune_entry* out, int32_t max, int32_t* n);

/*
 * Conservation totals of a state the caller owns, computed without allocating anything.
 * No counterpart in the reference.
 *
 * For callers that cannot let a library allocate device memory: a host that keeps all of its
 * GPU memory in its own pool or fixed arena and accounts for every byte (a serving process
 * admitting work against a fixed HBM budget), or a binding handed device buffers by another
 * runtime with no allocator of its own to call. It makes no cudaMalloc, cudaFree or other
 * allocating call; its scratch is a file-scope device array of SHZ_TOTALS_MAX_BLOCKS rows of
 * SHZ_DIAG_VALUES doubles (576 KiB) that every GPU loading the library holds until exit.
 *
 * cfg:    grid size n[3], dx, gamma, rho_floor, p_floor and device are read; the rest is ignored.
 *         States of more than SHZ_TOTALS_MAX_BLOCKS * SHZ_TOTALS_CELLS_PER_BLOCK cells
 *         (134,217,728 = 512^3) are refused with SHZ_E_CONFIG.
 * u1, u2: device pointers to the state, two float4 arrays in the layout above.
 * out:    device pointer to SHZ_DIAG_VALUES doubles: mass, momentum x/y/z, e_kin, e_int, e_tot,
 *         floored cells, max Mach (the fields of shz_diag, same meaning).
 * stream: cudaStream_t to enqueue on (NULL for the default stream); the call returns once the
 *         work is enqueued, and `out` is ready when the stream reaches it.
 *
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture. The address is kept per
 * device together with the id of the context it was found in: after a device reset
 * (cudaDeviceReset) the next call finds the new context and looks the address up again. The call
 * makes `device` current for its own work and puts the caller's current device back before it
 * returns. All calls share the one array: calls whose work overlaps on the GPU race on it, so
 * serialise them (one stream, or events between streams). Each call overwrites every row it
 * reads, so nothing left by an earlier call matters. On failure, shz_totals_noalloc_error() gives
 * the message of the calling thread's last failure.
 */
#define SHZ_DIAG_VALUES 9
#define SHZ_TOTALS_MAX_BLOCKS 8192
#define SHZ_TOTALS_CELLS_PER_BLOCK 16384
int shz_totals_noalloc(const shz_config* cfg, const void* u1, const void* u2, double* out, void* stream);
const char* shz_totals_noalloc_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SHADEROUS_B200_H */
