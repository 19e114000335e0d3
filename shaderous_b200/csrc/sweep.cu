// The uniform-grid hydro step as one fused kernel per step, plus its clock, rate and
// diagnostics kernels.
//
// One step of the reference (src/sim.ts:3187-3328 encodeSteps) is four passes: rates
// (hydro/rates.wgsl), the dt reduction and clock (gpu/reduce.wgsl, hydro/clock.wgsl), the
// Hancock predictor (hydro/predict.wgsl -> predictor.wgsl) and the update
// (hydro/update.wgsl -> tile.wgsl, flux.wgsl, riemann/hllc.wgsl, advance.wgsl, dual_energy.wgsl).
// Here a step is clock_kernel (one thread: dt from the last sweep's rate maximum, the float64
// clock advanced) and sweep_kernel, which reads each cell's conserved state once and in one
// pass recovers primitives, forms limited edge increments, takes the Hancock half step, solves
// each face's Riemann problem once, applies the conservative update with the dual-energy
// switch, writes the new state, and folds the new state's signal rate into the next step's
// maximum (warp shuffles, then one atomicMax per CTA on the float's bits).
//
// Decomposition: a CTA owns a TX x TY column of cells and marches it along z through tz planes
// (2.5D). Its threads are the (TX+2) x (TY+2) cells of the column plus one ring of halo cells.
// The primitives of the planes the predictor's z stencil reads sit in a ring of planes in shared
// memory, each plane the column plus the stencil's halo (as pairs: rho vx, vy vz, p s, one
// 8-byte load each), converted from the conserved state that a tiled TMA copy staged while the
// previous plane was computed. The z face below a cell and the running flux sums stay in the
// thread's registers; the face states toward the upper x and y faces go to shared memory so that
// the next thread can solve its lower face, and the x and y fluxes so that both cells read them
// (two float4 a thread and face). Each face flux is computed once and used by both cells, so both
// sides see bit-identical fluxes (the reference's flux-determinism check,
// src/validation/tests.ts:961).
//
// The arithmetic follows the reference's CPU scheme, src/reference/hydro.ts (RefHydro), in
// float32: a cell beyond a boundary takes the half-step state and flags of the cell it maps to
// (mirrored for a reflecting wall) with edge increments recomputed at the ghost position
// (hydro.ts:329-358). Collapsed axes (n = 1) carry no faces: in the reference their two faces
// carry equal fluxes that cancel.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "hydro_cell.cuh"
#include "hydro_math.cuh"
#include "diag_ext.cuh"
#include "sweep.h"
#include "tma.cuh"

namespace shz {

template <int DIM, int RECON>
struct Geo {
  static constexpr int H = (RECON == R_PPM) ? 3 : 2;   // halo of the primitives' region
  static constexpr int ZH = (RECON == R_PPM) ? 2 : 1;  // planes each way the predictor reads along z
  // 16 x 12 columns (8 warps a CTA): in 3D two CTAs leave 128 registers a thread (below); in 2D
  // three CTAs fit per SM at the 2D kernel's 72 registers (two of 16 x 16 did: 10-13 % slower)
  static constexpr int TX = (DIM == 1) ? 126 : 16;
  static constexpr int TY = (DIM == 1) ? 1 : 12;
  static constexpr int PX = TX + 2;
  static constexpr int PY = (DIM >= 2) ? TY + 2 : 1;
  static constexpr int NT = PX * PY;
  static constexpr int PN = PX * PY;
  static constexpr int WX = TX + 2 * H;
  static constexpr int WY = (DIM >= 2) ? TY + 2 * H : 1;
  static constexpr int WN = WX * WY;
  static constexpr int WC = 6;                               // primitives kept per cell (no sound speed)
  static constexpr int NBUF = (DIM == 3) ? 2 * ZH + 1 : 1;   // ring of planes: the predictor's z stencil
  static constexpr int NF = (DIM >= 2) ? 2 : 1;              // in-plane face directions
  // Registers per thread such that two CTAs are resident per SM (three in 2D). Warps are spread
  // over the SM's four sub-partitions, each with a 16K-register file: three 8-warp CTAs (2D) put 6
  // warps on one, and 6 x 32 x 80 <= 16384; two (3D) put 4, and 4 x 32 x 128 = 16384. The 3D sweep
  // needs the registers more than the wider columns: at 80 it spilled, and 16 x 12 columns with
  // 128 registers ran 6 % faster than 16 x 16 with 80 (the PPM Taylor-Green vortex at 512^3).
  static constexpr int MAXREG = (DIM == 1) ? 64 : (DIM == 3) ? 128 : 80;
  static constexpr size_t BASE_FLOATS = (size_t)NBUF * WC * WN + (size_t)NF * 8 * PN + (size_t)NF * 8 * PN + 32;
  // 3D: a staging area for one plane's conserved state, u1 box then u2 box (float4, x fastest),
  // filled by a tiled TMA copy; both boxes start on 128-byte boundaries.
  static constexpr size_t STAGE_OFS = (BASE_FLOATS + 31) / 32 * 32;
  static constexpr size_t STAGE_BOX = ((size_t)4 * WN + 31) / 32 * 32;
  static constexpr size_t SMEM_FLOATS = (DIM == 3) ? STAGE_OFS + 2 * STAGE_BOX : BASE_FLOATS;
  static constexpr size_t SMEM_BYTES = SMEM_FLOATS * sizeof(float);
};

// Primitives of one plane of the CTA's region (column plus stencil halo) into shared memory,
// through the boundary mapping.
template <int DIM, int RECON>
__device__ __forceinline__ void load_w_plane(const KParams& P, const float4* __restrict__ u1, const float4* __restrict__ u2,
                                             int x0, int y0, int plane, float* __restrict__ sWb) {
  using G = Geo<DIM, RECON>;
  float fz = 1.f;
  // (a halo face's ghost planes are stored beyond the slab: read as they are)
  const bool zhalo = (DIM == 3) && ((plane < 0 && P.bc_lo[2] == BC_HALO) || (plane >= P.n[2] && P.bc_hi[2] == BC_HALO));
  const int gz = (DIM == 3) ? (zhalo ? plane : bc_map(plane, P.n[2], P.bc_lo[2], P.bc_hi[2], fz)) : 0;
  const ptrdiff_t zoff = (ptrdiff_t)gz * P.n[1] * P.n[0];
  for (int idx = threadIdx.x; idx < G::WN; idx += G::NT) {
    const int lx = idx % G::WX, ly = idx / G::WX;
    float fx, fy = 1.f;
    const int gx = bc_map(x0 - G::H + lx, P.n[0], P.bc_lo[0], P.bc_hi[0], fx);
    const int gy = (DIM >= 2) ? bc_map(y0 - G::H + ly, P.n[1], P.bc_lo[1], P.bc_hi[1], fy) : 0;
    const ptrdiff_t o = zoff + (ptrdiff_t)gy * P.n[0] + gx;
    const float4 a = __ldg(u1 + o), b = __ldg(u2 + o);
    float w[6];
    prim6_from_cons(a, b, P, fx, fy, fz, w);
#pragma unroll
    for (int c = 0; c < 3; c++) reinterpret_cast<float2*>(sWb)[c * G::WN + idx] = make_float2(w[2 * c], w[2 * c + 1]);
  }
}

// The six stored primitives of region cell (wx, wy) of a plane.
template <int DIM, int RECON>
__device__ __forceinline__ void read_w(const float* __restrict__ sWb, int wx, int wy, float* w) {
  using G = Geo<DIM, RECON>;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float2 t = reinterpret_cast<const float2*>(sWb)[c * G::WN + wy * G::WX + wx];
    w[2 * c] = t.x;
    w[2 * c + 1] = t.y;
  }
}

__device__ __forceinline__ void unpack7(const float4 a, const float4 b, float* f) {
  f[0] = a.x;
  f[1] = a.y;
  f[2] = a.z;
  f[3] = a.w;
  f[4] = b.x;
  f[5] = b.y;
  f[6] = b.z;
}
__device__ __forceinline__ void unpack8(const float4 a, const float4 b, float* f) {
  unpack7(a, b, f);
  f[7] = b.w;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block maximum of a non-negative rate into *out (as the float's bits: non-negative floats
// order as unsigned integers). fmaxf drops NaN operands, so rate_guard carries a NaN rate as
// +inf, which orders above every finite rate and which the clock reports.
template <int NT>
__device__ __forceinline__ void block_max_to(float v, float* sRed, unsigned* out) {
  v = warp_max(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sRed[warp] = v;
  __syncthreads();
  if (warp == 0) {
    constexpr int NW = (NT + 31) / 32;
    float m = lane < NW ? sRed[lane] : 0.f;
    m = warp_max(m);
    if (lane == 0) atomicMax(out, __float_as_uint(m));
  }
}

__device__ __forceinline__ float rate_guard(float r) { return (r == r) ? r : __int_as_float(0x7f800000); }

template <int DIM, int RECON, bool ISEN>
__global__ void __launch_bounds__(Geo<DIM, RECON>::NT) __maxnreg__((Geo<DIM, RECON>::MAXREG))
    sweep_kernel(const KParams P, const float4* __restrict__ u1, const float4* __restrict__ u2, float4* __restrict__ o1,
                 float4* __restrict__ o2, const DevClock* __restrict__ clk, unsigned* __restrict__ rate_out, int tz,
                 const __grid_constant__ CUtensorMap tm1, const __grid_constant__ CUtensorMap tm2, int zofs, int use_tma,
                 int* __restrict__ err) {
  using G = Geo<DIM, RECON>;
  constexpr int H = G::H, ZH = G::ZH, PX = G::PX, PN = G::PN, WN = G::WN, WC = G::WC;
  extern __shared__ __align__(128) float smem[];
  float* sW = smem;
  // face states and fluxes as two float4 a thread per face direction (k = 0 x, 1 y): entries
  // (2k) * PN + tid and (2k + 1) * PN + tid
  float4* sFace = reinterpret_cast<float4*>(sW + G::NBUF * WC * WN);
  float4* sFlux = sFace + G::NF * 2 * PN;
  float* sRed = reinterpret_cast<float*>(sFlux + G::NF * 2 * PN);

  const int tid = threadIdx.x;
  const int tx = tid % PX, ty = tid / PX;
  const int x0 = blockIdx.x * G::TX, y0 = blockIdx.y * G::TY;
  const int gx = x0 - 1 + tx, gy = (DIM >= 2) ? y0 - 1 + ty : 0;
  const int wx = tx + H - 1, wy = (DIM >= 2) ? ty + H - 1 : 0;
  const int wo = wy * G::WX + wx;  // own cell within a plane of the region
  const int nx = P.n[0], ny = P.n[1], nz = P.n[2];
  // Roles: tile_t updates cell (gx, gy); row_t / col_t: the row / column lies in the tile.
  const bool row_t = (DIM < 2) || (ty >= 1 && ty <= G::TY && gy < ny);
  const bool col_t = tx >= 1 && tx <= G::TX && gx < nx;
  const bool tile_t = row_t && col_t;
  const bool xface_t = row_t && tx >= 1 && tx <= G::TX + 1 && gx <= nx;  // solves the x face below gx
  const bool yface_t = (DIM >= 2) && col_t && ty >= 1 && ty <= G::TY + 1 && gy <= ny;

  const double dt = clk->dt;
  const float dtdx = (float)(dt / P.dx);
  const float h = (float)((0.5 * dt) / P.dx);
  float rate_max = 0.f;

  // A step held at the stop time (dt = 0) leaves the state as it is (clock.wgsl:120-125).
  if (clk->held) {
    const int zb = (DIM == 3) ? blockIdx.z * tz : 0;
    const int ze = (DIM == 3) ? min(zb + tz, nz) : 1;
    for (int idx = tid; idx < G::TX * G::TY; idx += G::NT) {
      const int cx = x0 + idx % G::TX, cy = (DIM >= 2) ? y0 + idx / G::TX : 0;
      if (cx >= nx || cy >= ny) continue;
      for (int z = zb; z < ze; z++) {
        const size_t o = ((size_t)z * ny + cy) * nx + cx;
        const float4 a = u1[o], b = u2[o];
        o1[o] = a;
        o2[o] = b;
        rate_max = fmaxf(rate_max, rate_guard(signal_rate(a, b, P)));
      }
    }
    block_max_to<G::NT>(rate_max, sRed, rate_out);
    return;
  }

  // Ghost cells across an outflow or reflecting x/y boundary take their half-step state from
  // the adjacent inner cell (hydro.ts:335-342); whether this CTA has any is CTA-uniform.
  const bool xg_lo = x0 == 0 && P.bc_lo[0] != 0;
  const bool xg_hi = x0 + G::TX >= nx && P.bc_hi[0] != 0;
  const bool yg_lo = (DIM >= 2) && y0 == 0 && P.bc_lo[1] != 0;
  const bool yg_hi = (DIM >= 2) && y0 + G::TY >= ny && P.bc_hi[1] != 0;
  const bool xyg = xg_lo || xg_hi || yg_lo || yg_hi;
  int g_src = -1, g_axis = 0;
  bool g_flip = false;
  if (xg_lo && gx == -1 && row_t) { g_src = tid + 1; g_axis = 0; g_flip = P.bc_lo[0] == 2; }
  if (xg_hi && gx == nx && row_t) { g_src = tid - 1; g_axis = 0; g_flip = P.bc_hi[0] == 2; }
  if (DIM >= 2 && yg_lo && gy == -1 && col_t) { g_src = tid + PX; g_axis = 1; g_flip = P.bc_lo[1] == 2; }
  if (DIM >= 2 && yg_hi && gy == ny && col_t) { g_src = tid - PX; g_axis = 1; g_flip = P.bc_hi[1] == 2; }

  const int z0 = (DIM == 3) ? blockIdx.z * tz : 0;
  const int z1 = (DIM == 3) ? min(z0 + tz, nz) : 1;
  // plane -> its slot of the ring (planes may be negative near the lower boundary)
  auto ring = [&](int plane) -> float* {
    return sW + (((plane % G::NBUF) + G::NBUF) % G::NBUF) * WC * WN;
  };

  float zhi_prev[7];      // face state below the upper z face of plane j-1
  float q_prev[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float flag_prev = 0.f;
  bool fo_prev = false;
  float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float ph_prev = 0.f;
  float gsu[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // edges of the lower z ghost (outflow / reflect)
  // CTA-uniform: a cell of plane j - 1 (column and halo ring) is shock-flagged. The faces of plane
  // j see the flags of planes j - 1 and j only; without any, the solver skips the HLL flux.
  bool flagged_prev = true;
#pragma unroll
  for (int v = 0; v < 7; v++) zhi_prev[v] = 0.f;

  // 3D columns whose stencil region lies inside the grid in x and y stage each plane's state with
  // one tiled TMA copy per array (boxes of WX x WY float4 at (x0 - H, y0 - H), the plane mapped
  // through the z boundary) while the previous plane is computed; columns at an x or y face keep
  // the per-cell loads through the boundary mapping.
  // (the staging boxes must start on 128-byte boundaries of shared memory; checked, not assumed)
  const bool tma_tile = (DIM == 3) && use_tma && x0 - H >= 0 && x0 - H + G::WX <= nx && y0 - H >= 0 &&
                        y0 - H + G::WY <= ny && (tma::smem_u32(smem + G::STAGE_OFS) & 127u) == 0;
  __shared__ __align__(8) uint64_t sBarU;
  const float4* stage1 = reinterpret_cast<const float4*>(smem + G::STAGE_OFS);
  const float4* stage2 = reinterpret_cast<const float4*>(smem + G::STAGE_OFS + G::STAGE_BOX);
  uint32_t uphase = 0;
  float stage_fz = 1.f;  // velocity sign of the staged plane (a mirrored z ghost)
  auto issue_plane = [&](int pl) {
    float fz = 1.f;
    const bool zhalo = (pl < 0 && P.bc_lo[2] == BC_HALO) || (pl >= nz && P.bc_hi[2] == BC_HALO);
    const int gz = zhalo ? pl : bc_map(pl, nz, P.bc_lo[2], P.bc_hi[2], fz);
    stage_fz = fz;
    if (tid == 0) {
      tma::fence_proxy_async();
      tma::mbar_expect_tx(&sBarU, (uint32_t)(2 * WN * sizeof(float4)));
      tma::tile3d_g2s(smem + G::STAGE_OFS, &tm1, 4 * (x0 - H), y0 - H, gz + zofs, &sBarU);
      tma::tile3d_g2s(smem + G::STAGE_OFS + G::STAGE_BOX, &tm2, 4 * (x0 - H), y0 - H, gz + zofs, &sBarU);
    }
  };
  // Columns at an x or y face of the grid (whose region the tiled copy cannot map through the
  // boundary) stage their planes too: each thread copies its own texels of the plane after the
  // next into the staging area by asynchronous copies (cp.async, through the boundary mapping) and
  // converts them a plane later, so that the loads are in flight during a plane's work.
  auto stage_plane = [&](int pl) {
    float fz = 1.f;
    const bool zhalo = (pl < 0 && P.bc_lo[2] == BC_HALO) || (pl >= nz && P.bc_hi[2] == BC_HALO);
    const int gz = zhalo ? pl : bc_map(pl, nz, P.bc_lo[2], P.bc_hi[2], fz);
    stage_fz = fz;
    const ptrdiff_t zoff = (ptrdiff_t)gz * ny * nx;
    float4* s1 = reinterpret_cast<float4*>(smem + G::STAGE_OFS);
    float4* s2 = reinterpret_cast<float4*>(smem + G::STAGE_OFS + G::STAGE_BOX);
    for (int idx = tid; idx < WN; idx += G::NT) {
      const int lx = idx % G::WX, ly = idx / G::WX;
      float fx, fy;
      const int sx = bc_map(x0 - H + lx, nx, P.bc_lo[0], P.bc_hi[0], fx);
      const int sy = bc_map(y0 - H + ly, ny, P.bc_lo[1], P.bc_hi[1], fy);
      const ptrdiff_t o = zoff + (ptrdiff_t)sy * nx + sx;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tma::smem_u32(s1 + idx)), "l"(u1 + o) : "memory");
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tma::smem_u32(s2 + idx)), "l"(u2 + o) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  auto land_plane = [&](float* dst) {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    for (int idx = tid; idx < WN; idx += G::NT) {
      const int lx = idx % G::WX, ly = idx / G::WX;
      float fx, fy;
      bc_map(x0 - H + lx, nx, P.bc_lo[0], P.bc_hi[0], fx);
      bc_map(y0 - H + ly, ny, P.bc_lo[1], P.bc_hi[1], fy);
      float w[6];
      prim6_from_cons(stage1[idx], stage2[idx], P, fx, fy, stage_fz, w);
#pragma unroll
      for (int c = 0; c < 3; c++) reinterpret_cast<float2*>(dst)[c * WN + idx] = make_float2(w[2 * c], w[2 * c + 1]);
    }
  };
  if constexpr (DIM == 3) {
    if (tma_tile) {
      if (tid == 0) {
        tma::mbar_init(&sBarU, 1);
        tma::fence_mbar_init();
      }
      __syncthreads();
    }
    // the planes below the first that the predictor reads along z
    for (int pl = z0 - 1 - ZH; pl <= z0 - 2 + ZH; pl++) load_w_plane<DIM, RECON>(P, u1, u2, x0, y0, pl, ring(pl));
    if (tma_tile) issue_plane(z0 - 1 + ZH);
    else stage_plane(z0 - 1 + ZH);
  }

  const int jb = (DIM == 3) ? z0 - 1 : 0;
  const int je = (DIM == 3) ? z1 : 0;
  // PPM along z: each plane's limited slope of the column's cell is used by the planes below, at
  // and above it; it is formed once, when plane j + 1's is first needed, and carried up the march
  // (zs_m, zs_0: the slopes at planes j - 1 and j; both formed at the first plane).
  constexpr bool ZCARRY = RECON == R_PPM && DIM == 3;
  float zs_m[6], zs_0[6];
  bool zs_ready = false;
  // the ring slot of plane j, advanced with j (a plane k planes away from j is in slot sj + k,
  // wrapped), instead of two remainders by NBUF per access
  int sj = ((jb % G::NBUF) + G::NBUF) % G::NBUF;
  auto ringk = [&](int k) -> float* {
    int s = sj + k;
    s = s >= G::NBUF ? s - G::NBUF : s;
    s = s < 0 ? s + G::NBUF : s;
    return sW + s * WC * WN;
  };
  for (int j = jb; j <= je; j++, sj = (sj + 1 == G::NBUF) ? 0 : sj + 1) {
    // 1. primitives of plane j + ZH (the plane itself when there is no march)
    const int lp = (DIM == 3) ? j + ZH : 0;
    if (tma_tile) {
      const bool ok = tma::mbar_wait(&sBarU, uphase, tma::WAIT_LIMIT);
      uphase ^= 1u;
      if (__syncthreads_or(!ok)) {
        if (tid == 0 && err) atomicExch(err, tma::ERR_TMA_TIMEOUT);
        return;
      }
      float* dst = ringk((DIM == 3) ? ZH : 0);
      for (int idx = tid; idx < WN; idx += G::NT) {
        float w[6];
        prim6_from_cons(stage1[idx], stage2[idx], P, 1.f, 1.f, stage_fz, w);
#pragma unroll
        for (int c = 0; c < 3; c++) reinterpret_cast<float2*>(dst)[c * WN + idx] = make_float2(w[2 * c], w[2 * c + 1]);
      }
      __syncthreads();
      // the staging area is free again: the next plane's copy overlaps this plane's work
      if (j + 1 <= je) issue_plane(j + 1 + ZH);
    } else if constexpr (DIM == 3) {
      land_plane(ringk(ZH));
      if (j + 1 <= je) stage_plane(j + 1 + ZH);
      __syncthreads();
    } else {
      load_w_plane<DIM, RECON>(P, u1, u2, x0, y0, lp, ringk(0));
      __syncthreads();
    }
    const float* sWj = ringk(0);
    if constexpr (ZCARRY) {
      if (!zs_ready) {
        float c2[7], c1[7], a0[7], b1[7];
        read_w<DIM, RECON>(ringk(-2), wx, wy, c2);
        read_w<DIM, RECON>(ringk(-1), wx, wy, c1);
        read_w<DIM, RECON>(sWj, wx, wy, a0);
        read_w<DIM, RECON>(ringk(1), wx, wy, b1);
#pragma unroll
        for (int v = 0; v < 6; v++) {
          zs_m[v] = ppm_slope(c2[v], c1[v], a0[v]);
          zs_0[v] = ppm_slope(c1[v], a0[v], b1[v]);
        }
        zs_ready = true;
      }
    }
    // the z edge increments of this plane's cell (c; m, p below and above) from the carried
    // slopes and the new one at plane j + 1; the slopes then move up a plane
    auto z_edges = [&](const float* m, const float* c, const float* p, float* su_z, float* sd_z) {
      float p2v[6];
      read_w<DIM, RECON>(ringk(2), wx, wy, p2v);
#pragma unroll
      for (int v = 0; v < 6; v++) {
        const float zp = ppm_slope(c[v], p[v], p2v[v]);
        ppm_incs_d(m[v], c[v], p[v], zs_m[v], zs_0[v], zp, su_z[v], sd_z[v]);
        zs_m[v] = zs_0[v];
        zs_0[v] = zp;
      }
    };

    if constexpr (DIM == 3) {
      // The z ghost planes (outflow / reflect) need only their edges toward the domain, at the
      // ghost position; their half-step state is that of the adjacent inner plane.
      const bool zg_lo = j == -1 && bc_inner(P.bc_lo[2]);
      const bool zg_hi = j == nz && bc_inner(P.bc_hi[2]);
      if (zg_lo || zg_hi) {
        float c[7], m[7], p[7], m2[7], p2[7], su[6], sd[6];
        read_w<DIM, RECON>(sWj, wx, wy, c);
        with_cs(c, P);
        read_w<DIM, RECON>(ringk(-1), wx, wy, m);
        read_w<DIM, RECON>(ringk(1), wx, wy, p);
        if constexpr (ZCARRY) {
          (void)m2;
          (void)p2;
          z_edges(m, c, p, su, sd);
        } else {
          axis_edges<RECON, ISEN>(m2, m, c, p, p2, P.inv_gamma, su, sd);
        }
        if (zg_lo) {
#pragma unroll
          for (int v = 0; v < 6; v++) gsu[v] = su[v];
          flagged_prev = false;  // plane 0's faces see plane 0's flags only
        } else if (tile_t) {
          Pred g;
#pragma unroll
          for (int v = 0; v < 6; v++) g.q[v] = q_prev[v];
          if (P.bc_hi[2] == 2) g.q[3] = -g.q[3];
          g.flag = flag_prev;
          g.fo = fo_prev;
          float zlo[7], Fz[8];
          face_state(g, sd, -1.f, zlo);
          riemann<2>(zhi_prev, zlo, P, Fz, flagged_prev);
#pragma unroll
          for (int v = 0; v < 8; v++) acc[v] -= Fz[v];
          const size_t o = ((size_t)(j - 1) * ny + gy) * nx + gx;
          float4 na, nb;
          update_cell(__ldg(u1 + o), __ldg(u2 + o), acc, ph_prev, dtdx, P, na, nb);
          o1[o] = na;
          o2[o] = nb;
          rate_max = fmaxf(rate_max, rate_guard(signal_rate(na, nb, P)));
        }
        continue;
      }
    }

    // 2. predictor at plane j: edges per active axis, shock flag, Hancock half step.
    float c[7];
    read_w<DIM, RECON>(sWj, wx, wy, c);
    with_cs(c, P);
    float su[DIM][6], sd[DIM][6];
    float conv = 0.f, jump = -INFINITY;
    {
      float m[7], p[7], m2[7], p2[7];
      read_w<DIM, RECON>(sWj, wx - 1, wy, m);
      read_w<DIM, RECON>(sWj, wx + 1, wy, p);
      if constexpr (RECON == R_PPM) {
        read_w<DIM, RECON>(sWj, wx - 2, wy, m2);
        read_w<DIM, RECON>(sWj, wx + 2, wy, p2);
      }
      axis_edges<RECON, ISEN>(m2, m, c, p, p2, P.inv_gamma, su[0], sd[0]);
      conv += p[1] - m[1];
      jump = fmaxf(jump, jump_excess(m[4], p[4], P.shock_thresh));
      if constexpr (DIM >= 2) {
        read_w<DIM, RECON>(sWj, wx, wy - 1, m);
        read_w<DIM, RECON>(sWj, wx, wy + 1, p);
        if constexpr (RECON == R_PPM) {
          read_w<DIM, RECON>(sWj, wx, wy - 2, m2);
          read_w<DIM, RECON>(sWj, wx, wy + 2, p2);
        }
        axis_edges<RECON, ISEN>(m2, m, c, p, p2, P.inv_gamma, su[1], sd[1]);
        conv += p[2] - m[2];
        jump = fmaxf(jump, jump_excess(m[4], p[4], P.shock_thresh));
      }
      if constexpr (DIM == 3) {
        read_w<DIM, RECON>(ringk(-1), wx, wy, m);
        read_w<DIM, RECON>(ringk(1), wx, wy, p);
        if constexpr (ZCARRY) {
          z_edges(m, c, p, su[2], sd[2]);
        } else {
          axis_edges<RECON, ISEN>(m2, m, c, p, p2, P.inv_gamma, su[2], sd[2]);
        }
        conv += p[3] - m[3];
        jump = fmaxf(jump, jump_excess(m[4], p[4], P.shock_thresh));
      }
    }
    (void)wo;
    Pred pr;
    hancock<DIM>(c, conv, jump, su, sd, h, P, pr);

    const bool tile_plane = j >= z0 && j < z1;
    // 3. ghosts across outflow / reflecting x/y boundaries take the inner cell's half step.
    if (xyg && tile_plane) {
      sFlux[tid] = make_float4(pr.q[0], pr.q[1], pr.q[2], pr.q[3]);
      sFlux[PN + tid] = make_float4(pr.q[4], pr.q[5], pr.flag, pr.fo ? 1.f : 0.f);
      __syncthreads();
      if (g_src >= 0) {
        const float4 a = sFlux[g_src], b = sFlux[PN + g_src];
        pr.q[0] = a.x;
        pr.q[1] = a.y;
        pr.q[2] = a.z;
        pr.q[3] = a.w;
        pr.q[4] = b.x;
        pr.q[5] = b.y;
        pr.flag = b.z;
        pr.fo = b.w != 0.f;
        if (g_flip) pr.q[1 + g_axis] = -pr.q[1 + g_axis];
      }
    }
    if constexpr (DIM == 3) {
      // plane 0 stands in for the lower z ghost: its face state toward plane 0
      if (j == 0 && bc_inner(P.bc_lo[2])) {
        Pred g = pr;
        if (P.bc_lo[2] == 2) g.q[3] = -g.q[3];
        face_state(g, gsu, 1.f, zhi_prev);
      }
    }

    // 4. face states toward the upper x and y faces, for the thread beyond each.
    if (tile_plane) {
      float f[7];
      face_state(pr, su[0], 1.f, f);
      sFace[tid] = make_float4(f[0], f[1], f[2], f[3]);
      sFace[PN + tid] = make_float4(f[4], f[5], f[6], 0.f);
      if constexpr (DIM >= 2) {
        face_state(pr, su[1], 1.f, f);
        sFace[2 * PN + tid] = make_float4(f[0], f[1], f[2], f[3]);
        sFace[3 * PN + tid] = make_float4(f[4], f[5], f[6], 0.f);
      }
    }
    const bool flagged = __syncthreads_or(pr.flag != 0.f);
    const bool hll_any = flagged || (DIM == 3 && flagged_prev);
    flagged_prev = flagged;

    // 5. fluxes: the lower x and y faces into shared memory, the lower z face in registers.
    if (tile_plane) {
      if (xface_t) {
        float L[7], R[7], F[8];
        unpack7(sFace[tid - 1], sFace[PN + tid - 1], L);
        face_state(pr, sd[0], -1.f, R);
        riemann<0>(L, R, P, F, hll_any);
        sFlux[tid] = make_float4(F[0], F[1], F[2], F[3]);
        sFlux[PN + tid] = make_float4(F[4], F[5], F[6], F[7]);
      }
      if constexpr (DIM >= 2) {
        if (yface_t) {
          float L[7], R[7], F[8];
          unpack7(sFace[2 * PN + tid - PX], sFace[3 * PN + tid - PX], L);
          face_state(pr, sd[1], -1.f, R);
          riemann<1>(L, R, P, F, hll_any);
          sFlux[2 * PN + tid] = make_float4(F[0], F[1], F[2], F[3]);
          sFlux[3 * PN + tid] = make_float4(F[4], F[5], F[6], F[7]);
        }
      }
    }
    float Fz[8];
    if constexpr (DIM == 3) {
      if (tile_t && j >= z0) {
        float R[7];
        face_state(pr, sd[2], -1.f, R);
        riemann<2>(zhi_prev, R, P, Fz, hll_any);
      }
    }
    __syncthreads();

    // 6. updates: plane j-1 now has its upper z flux; plane j gets its in-plane fluxes.
    if (tile_t) {
      if constexpr (DIM == 3) {
        if (j - 1 >= z0) {
#pragma unroll
          for (int v = 0; v < 8; v++) acc[v] -= Fz[v];
          const size_t o = ((size_t)(j - 1) * ny + gy) * nx + gx;
          float4 na, nb;
          update_cell(__ldg(u1 + o), __ldg(u2 + o), acc, ph_prev, dtdx, P, na, nb);
          o1[o] = na;
          o2[o] = nb;
          rate_max = fmaxf(rate_max, rate_guard(signal_rate(na, nb, P)));
        }
      }
      if (tile_plane) {
        float xl[8], xu[8], yl[8], yu[8];
        unpack8(sFlux[tid], sFlux[PN + tid], xl);
        unpack8(sFlux[tid + 1], sFlux[PN + tid + 1], xu);
        if constexpr (DIM >= 2) {
          unpack8(sFlux[2 * PN + tid], sFlux[3 * PN + tid], yl);
          unpack8(sFlux[2 * PN + tid + PX], sFlux[3 * PN + tid + PX], yu);
        }
#pragma unroll
        for (int v = 0; v < 8; v++) {
          float a = xl[v];
          a -= xu[v];
          if constexpr (DIM >= 2) {
            a += yl[v];
            a -= yu[v];
          }
          if constexpr (DIM == 3) a += Fz[v];
          acc[v] = a;
        }
        ph_prev = pr.q[4];
        if constexpr (DIM < 3) {
          const size_t o = (size_t)gy * nx + gx;
          float4 na, nb;
          update_cell(__ldg(u1 + o), __ldg(u2 + o), acc, ph_prev, dtdx, P, na, nb);
          o1[o] = na;
          o2[o] = nb;
          rate_max = fmaxf(rate_max, rate_guard(signal_rate(na, nb, P)));
        }
      }
    }
    if constexpr (DIM == 3) {
      face_state(pr, su[2], 1.f, zhi_prev);
#pragma unroll
      for (int v = 0; v < 6; v++) q_prev[v] = pr.q[v];
      flag_prev = pr.flag;
      fo_prev = pr.fo;
    }
  }
  block_max_to<G::NT>(rate_max, sRed, rate_out);
}

// ---------------------------------------------------------------------------------------------
// The 2D step as a march along y. A CTA owns a row segment of TX cells and marches it up through
// `rows` rows, as the 3D sweep marches its columns along z: its threads are the segment's cells
// plus one halo cell at each end, the primitives of the rows the predictor reads along y sit in a
// ring of rows in shared memory, the state of the row after the next is in flight into a staging
// row (asynchronous copies, a row ahead of its conversion), and the y face below a cell and the
// running flux sums stay in the thread's registers. Against the 2D tile form (16 x 12 cells with a
// ring of halo cells) it runs the predictor 1.02 times per cell instead of 1.31 and converts each
// row once. The arithmetic per cell is the same functions in the same order; the two kernels agree
// to rounding (the compiler may contract a multiply and an add differently in each).
template <int RECON>
struct RowGeo {
  static constexpr int H = (RECON == R_PPM) ? 3 : 2;   // halo of a row of primitives
  static constexpr int ZH = (RECON == R_PPM) ? 2 : 1;  // rows each way the predictor reads along y
  static constexpr int TX = 126;                       // cells of a CTA's row segment
  static constexpr int PX = TX + 2;                    // threads: the segment and a halo cell each end
  static constexpr int NT = PX;
  static constexpr int WX = TX + 2 * H;                // texels of a row of primitives
  static constexpr int WC = 6;
  static constexpr int NBUF = 2 * ZH + 1;
  // the ring, the x face states and fluxes, the staging row (u1 then u2 of WX texels), the reduction
  static constexpr size_t STAGE_OFS = (size_t)NBUF * WC * WX + (size_t)2 * 4 * PX + (size_t)2 * 4 * PX;
  static constexpr size_t SMEM_FLOATS = STAGE_OFS + (size_t)2 * 4 * WX + 32;
  static constexpr size_t SMEM_BYTES = SMEM_FLOATS * sizeof(float);
  static_assert((NBUF * WC * WX) % 4 == 0, "the face states start on a 16-byte boundary");
};

// Primitives of row r of the segment's region (through the y and x boundary mappings) into a ring
// slot: float2 pairs (rho vx, vy vz, p s), as the 3D sweep's planes.
template <int RECON>
__device__ __forceinline__ void load_w_row(const KParams& P, const float4* __restrict__ u1, const float4* __restrict__ u2,
                                           int x0, int r, float* __restrict__ dst) {
  using G = RowGeo<RECON>;
  float fy;
  const int gy = bc_map(r, P.n[1], P.bc_lo[1], P.bc_hi[1], fy);
  const ptrdiff_t yoff = (ptrdiff_t)gy * P.n[0];
  for (int idx = threadIdx.x; idx < G::WX; idx += G::NT) {
    float fx;
    const int gx = bc_map(x0 - G::H + idx, P.n[0], P.bc_lo[0], P.bc_hi[0], fx);
    const float4 a = __ldg(u1 + yoff + gx), b = __ldg(u2 + yoff + gx);
    float w[6];
    prim6_from_cons(a, b, P, fx, fy, 1.f, w);
#pragma unroll
    for (int c = 0; c < 3; c++) reinterpret_cast<float2*>(dst)[c * G::WX + idx] = make_float2(w[2 * c], w[2 * c + 1]);
  }
}

template <int RECON>
__device__ __forceinline__ void read_row(const float* __restrict__ sWr, int wx, float* w) {
  using G = RowGeo<RECON>;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float2 t = reinterpret_cast<const float2*>(sWr)[c * G::WX + wx];
    w[2 * c] = t.x;
    w[2 * c + 1] = t.y;
  }
}

template <int RECON, bool ISEN>
// (5 CTAs of 4 warps per SM: 96 registers a thread; at 128 and 4 CTAs, or at 80 and 6 with spills,
// the Kelvin-Helmholtz march ran 4-8 % slower)
__global__ void __launch_bounds__(RowGeo<RECON>::NT, 5)
    sweep_rows_kernel(const KParams P, const float4* __restrict__ u1, const float4* __restrict__ u2,
                      float4* __restrict__ o1, float4* __restrict__ o2, const DevClock* __restrict__ clk,
                      unsigned* __restrict__ rate_out, int rows) {
  using G = RowGeo<RECON>;
  constexpr int H = G::H, ZH = G::ZH, PX = G::PX, WX = G::WX, WC = G::WC;
  extern __shared__ __align__(128) float smem[];
  float* sW = smem;
  float4* sFace = reinterpret_cast<float4*>(sW + G::NBUF * WC * WX);  // upper x face states, 2 a thread
  float4* sFlux = sFace + 2 * PX;                                     // lower x face fluxes, 2 a thread
  float4* sStage = reinterpret_cast<float4*>(smem + G::STAGE_OFS);  // the next row's state, in flight
  float* sRed = smem + G::STAGE_OFS + 2 * 4 * WX;

  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * G::TX;
  const int gx = x0 - 1 + tid;
  const int wx = tid + H - 1;
  const int nx = P.n[0], ny = P.n[1];
  const bool col_t = tid >= 1 && tid <= G::TX && gx < nx;             // updates cell gx
  const bool xface_t = tid >= 1 && tid <= G::TX + 1 && gx <= nx;       // solves the x face below gx
  const int y0 = blockIdx.y * rows, y1 = min(y0 + rows, ny);

  const double dt = clk->dt;
  const float dtdx = (float)(dt / P.dx);
  const float h = (float)((0.5 * dt) / P.dx);
  float rate_max = 0.f;

  if (clk->held) {
    if (col_t)
      for (int y = y0; y < y1; y++) {
        const size_t o = (size_t)y * nx + gx;
        const float4 a = u1[o], b = u2[o];
        o1[o] = a;
        o2[o] = b;
        rate_max = fmaxf(rate_max, rate_guard(signal_rate(a, b, P)));
      }
    block_max_to<G::NT>(rate_max, sRed, rate_out);
    return;
  }

  // x ghosts across an outflow or reflecting face take the inner cell's half step (hydro.ts:335-342)
  const bool xg_lo = x0 == 0 && P.bc_lo[0] != 0;
  const bool xg_hi = x0 + G::TX >= nx && P.bc_hi[0] != 0;
  const bool xg = xg_lo || xg_hi;
  int g_src = -1;
  bool g_flip = false;
  if (xg_lo && gx == -1) { g_src = tid + 1; g_flip = P.bc_lo[0] == 2; }
  if (xg_hi && gx == nx) { g_src = tid - 1; g_flip = P.bc_hi[0] == 2; }

  float yhi_prev[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // face state below the upper y face of row j-1
  float q_prev[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float flag_prev = 0.f;
  bool fo_prev = false;
  float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float ph_prev = 0.f;
  float gsu[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // edges of the lower y ghost (outflow / reflect)
  bool flagged_prev = true;  // CTA-uniform: a cell of row j - 1 is shock-flagged

  const int jb = y0 - 1, je = y1;
  int sj = ((jb % G::NBUF) + G::NBUF) % G::NBUF;  // the ring slot of row j
  auto ringk = [&](int k) -> float* {
    int sl = sj + k;
    sl = sl >= G::NBUF ? sl - G::NBUF : sl;
    sl = sl < 0 ? sl + G::NBUF : sl;
    return sW + sl * WC * WX;
  };
  for (int r = jb - ZH; r <= jb - 1 + ZH; r++) {
    int sl = ((r % G::NBUF) + G::NBUF) % G::NBUF;
    load_w_row<RECON>(P, u1, u2, x0, r, sW + sl * WC * WX);
  }
  // Row r's state into the staging row by asynchronous copies (each thread its own texels), a row
  // ahead of its conversion, so that the loads are in flight during a row's work.
  auto stage_row = [&](int r) {
    float fy;
    const int gy = bc_map(r, ny, P.bc_lo[1], P.bc_hi[1], fy);
    for (int idx = tid; idx < WX; idx += G::NT) {
      float fx;
      const int gxx = bc_map(x0 - H + idx, nx, P.bc_lo[0], P.bc_hi[0], fx);
      const size_t o = (size_t)gy * nx + gxx;
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tma::smem_u32(sStage + idx)), "l"(u1 + o) : "memory");
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tma::smem_u32(sStage + WX + idx)), "l"(u2 + o)
                   : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // the staged row r (this thread's copies landed) converted into a ring slot
  auto land_row = [&](int r, float* dst) {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    float fy;
    bc_map(r, ny, P.bc_lo[1], P.bc_hi[1], fy);
    for (int idx = tid; idx < WX; idx += G::NT) {
      float fx;
      bc_map(x0 - H + idx, nx, P.bc_lo[0], P.bc_hi[0], fx);
      float w[6];
      prim6_from_cons(sStage[idx], sStage[WX + idx], P, fx, fy, 1.f, w);
#pragma unroll
      for (int c = 0; c < 3; c++) reinterpret_cast<float2*>(dst)[c * WX + idx] = make_float2(w[2 * c], w[2 * c + 1]);
    }
  };
  stage_row(jb + ZH);
  // PPM along y: slopes carried up the march (ys_m, ys_0 at rows j - 1 and j)
  constexpr bool YCARRY = RECON == R_PPM;
  float ys_m[6], ys_0[6];
  bool ys_ready = false;
  for (int j = jb; j <= je; j++, sj = (sj + 1 == G::NBUF) ? 0 : sj + 1) {
    land_row(j + ZH, ringk(ZH));
    if (j + 1 <= je) stage_row(j + 1 + ZH);
    __syncthreads();
    const float* sWj = ringk(0);
    if constexpr (YCARRY) {
      if (!ys_ready) {
        float c2[6], c1[6], a0[6], b1[6];
        read_row<RECON>(ringk(-2), wx, c2);
        read_row<RECON>(ringk(-1), wx, c1);
        read_row<RECON>(sWj, wx, a0);
        read_row<RECON>(ringk(1), wx, b1);
#pragma unroll
        for (int v = 0; v < 6; v++) {
          ys_m[v] = ppm_slope(c2[v], c1[v], a0[v]);
          ys_0[v] = ppm_slope(c1[v], a0[v], b1[v]);
        }
        ys_ready = true;
      }
    }
    auto y_edges = [&](const float* m, const float* c, const float* p, float* su_y, float* sd_y) {
      float p2v[6];
      read_row<RECON>(ringk(2), wx, p2v);
#pragma unroll
      for (int v = 0; v < 6; v++) {
        const float yp = ppm_slope(c[v], p[v], p2v[v]);
        ppm_incs_d(m[v], c[v], p[v], ys_m[v], ys_0[v], yp, su_y[v], sd_y[v]);
        ys_m[v] = ys_0[v];
        ys_0[v] = yp;
      }
    };

    // The y ghost rows (outflow / reflect): their edges toward the domain at the ghost position;
    // their half step is that of the adjacent inner row.
    const bool yg_lo = j == -1 && bc_inner(P.bc_lo[1]);
    const bool yg_hi = j == ny && bc_inner(P.bc_hi[1]);
    if (yg_lo || yg_hi) {
      float c[7], m[7], p[7], m2[7], p2[7], su[6], sd[6];
      read_row<RECON>(sWj, wx, c);
      with_cs(c, P);
      read_row<RECON>(ringk(-1), wx, m);
      read_row<RECON>(ringk(1), wx, p);
      if constexpr (YCARRY) {
        (void)m2;
        (void)p2;
        y_edges(m, c, p, su, sd);
      } else {
        axis_edges<RECON, ISEN, false>(m2, m, c, p, p2, P.inv_gamma, su, sd);
      }
      if (yg_lo) {
#pragma unroll
        for (int v = 0; v < 6; v++) gsu[v] = su[v];
        flagged_prev = false;  // row 0's faces see row 0's flags only
      } else if (col_t) {
        Pred g;
#pragma unroll
        for (int v = 0; v < 6; v++) g.q[v] = q_prev[v];
        if (P.bc_hi[1] == 2) g.q[2] = -g.q[2];
        g.flag = flag_prev;
        g.fo = fo_prev;
        float ylo[7], Fy[8];
        face_state(g, sd, -1.f, ylo);
        riemann<1>(yhi_prev, ylo, P, Fy, flagged_prev);
#pragma unroll
        for (int v = 0; v < 8; v++) acc[v] -= Fy[v];
        const size_t o = (size_t)(j - 1) * nx + gx;
        float4 na, nb;
        update_cell(__ldg(u1 + o), __ldg(u2 + o), acc, ph_prev, dtdx, P, na, nb);
        o1[o] = na;
        o2[o] = nb;
        rate_max = fmaxf(rate_max, rate_guard(signal_rate(na, nb, P)));
      }
      continue;
    }

    // predictor at row j
    float c[7];
    read_row<RECON>(sWj, wx, c);
    with_cs(c, P);
    float su[2][6], sd[2][6];
    float conv = 0.f, jump = -INFINITY;
    {
      float m[7], p[7], m2[7], p2[7];
      read_row<RECON>(sWj, wx - 1, m);
      read_row<RECON>(sWj, wx + 1, p);
      if constexpr (RECON == R_PPM) {
        read_row<RECON>(sWj, wx - 2, m2);
        read_row<RECON>(sWj, wx + 2, p2);
      }
      axis_edges<RECON, ISEN, false>(m2, m, c, p, p2, P.inv_gamma, su[0], sd[0]);
      conv += p[1] - m[1];
      jump = fmaxf(jump, jump_excess(m[4], p[4], P.shock_thresh));
      read_row<RECON>(ringk(-1), wx, m);
      read_row<RECON>(ringk(1), wx, p);
      if constexpr (YCARRY) {
        y_edges(m, c, p, su[1], sd[1]);
      } else {
        axis_edges<RECON, ISEN, false>(m2, m, c, p, p2, P.inv_gamma, su[1], sd[1]);
      }
      conv += p[2] - m[2];
      jump = fmaxf(jump, jump_excess(m[4], p[4], P.shock_thresh));
    }
    Pred pr;
    hancock<2>(c, conv, jump, su, sd, h, P, pr);

    const bool row_plane = j >= y0 && j < y1;
    if (xg && row_plane) {
      sFlux[tid] = make_float4(pr.q[0], pr.q[1], pr.q[2], pr.q[3]);
      sFlux[PX + tid] = make_float4(pr.q[4], pr.q[5], pr.flag, pr.fo ? 1.f : 0.f);
      __syncthreads();
      if (g_src >= 0) {
        const float4 a = sFlux[g_src], b = sFlux[PX + g_src];
        pr.q[0] = a.x;
        pr.q[1] = a.y;
        pr.q[2] = a.z;
        pr.q[3] = a.w;
        pr.q[4] = b.x;
        pr.q[5] = b.y;
        pr.flag = b.z;
        pr.fo = b.w != 0.f;
        if (g_flip) pr.q[1] = -pr.q[1];
      }
    }
    // row 0 stands in for the lower y ghost: its face state toward row 0
    if (j == 0 && bc_inner(P.bc_lo[1])) {
      Pred g = pr;
      if (P.bc_lo[1] == 2) g.q[2] = -g.q[2];
      face_state(g, gsu, 1.f, yhi_prev);
    }
    if (row_plane) {
      float f[7];
      face_state(pr, su[0], 1.f, f);
      sFace[tid] = make_float4(f[0], f[1], f[2], f[3]);
      sFace[PX + tid] = make_float4(f[4], f[5], f[6], 0.f);
    }
    const bool flagged = __syncthreads_or(pr.flag != 0.f);
    const bool hll_any = flagged || flagged_prev;
    flagged_prev = flagged;

    if (row_plane && xface_t) {
      float L[7], R[7], F[8];
      unpack7(sFace[tid - 1], sFace[PX + tid - 1], L);
      face_state(pr, sd[0], -1.f, R);
      riemann<0>(L, R, P, F, hll_any);
      sFlux[tid] = make_float4(F[0], F[1], F[2], F[3]);
      sFlux[PX + tid] = make_float4(F[4], F[5], F[6], F[7]);
    }
    float Fy[8];
    if (col_t && j >= y0) {
      float R[7];
      face_state(pr, sd[1], -1.f, R);
      riemann<1>(yhi_prev, R, P, Fy, hll_any);
    }
    __syncthreads();

    if (col_t) {
      if (j - 1 >= y0) {
#pragma unroll
        for (int v = 0; v < 8; v++) acc[v] -= Fy[v];
        const size_t o = (size_t)(j - 1) * nx + gx;
        float4 na, nb;
        update_cell(__ldg(u1 + o), __ldg(u2 + o), acc, ph_prev, dtdx, P, na, nb);
        o1[o] = na;
        o2[o] = nb;
        rate_max = fmaxf(rate_max, rate_guard(signal_rate(na, nb, P)));
      }
      if (row_plane) {
        float xl[8], xu[8];
        unpack8(sFlux[tid], sFlux[PX + tid], xl);
        unpack8(sFlux[tid + 1], sFlux[PX + tid + 1], xu);
#pragma unroll
        for (int v = 0; v < 8; v++) {
          float a = xl[v];
          a -= xu[v];
          a += Fy[v];
          acc[v] = a;
        }
        ph_prev = pr.q[4];
      }
    }
    face_state(pr, su[1], 1.f, yhi_prev);
#pragma unroll
    for (int v = 0; v < 6; v++) q_prev[v] = pr.q[v];
    flag_prev = pr.flag;
    fo_prev = pr.fo;
  }
  block_max_to<G::NT>(rate_max, sRed, rate_out);
}

// The signal-rate maximum of a state (the reference's rates pass, hydro/rates.wgsl, and its
// reduction, gpu/reduce.wgsl): used for the first step after the state is set.
__global__ void rate_kernel(const KParams P, const float4* __restrict__ u1, const float4* __restrict__ u2, size_t ncell,
                            unsigned* __restrict__ out) {
  __shared__ float sRed[32];
  float m = 0.f;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < ncell; o += (size_t)gridDim.x * blockDim.x)
    m = fmaxf(m, rate_guard(signal_rate(__ldg(u1 + o), __ldg(u2 + o), P)));
  block_max_to<256>(m, sRed, out);
}

// One thread: dt from the rate maximum (clock.wgsl:38-147, in the reference's CPU form
// hydro.ts:382 dt = min(cfl dx / rate, t_end - t)), the clock advanced by the step in float64.
// A rate that is NaN or infinite marks the clock bad and holds it.
__global__ void clock_kernel(DevClock* clk, unsigned* rates, int slot) {
  const float rate = __uint_as_float(rates[slot]);
  rates[slot ^ 1] = 0u;
  const double t = clk->t;
  double dt = clk->cfl_dx / fmax((double)rate, 1e-30);
  if (!(rate == rate) || isinf(rate)) clk->bad = 1;
  dt = fmin(dt, clk->dt_max);
  const double te = clk->t_end;
  if (te < HUGE_VAL) {
    const double rem = te - t;
    if (rem <= 1e-12 * fabs(te)) dt = 0.0;
    else dt = fmin(dt, rem);
  }
  if (clk->bad) dt = 0.0;
  clk->dt = dt;
  clk->held = dt > 0.0 ? 0 : 1;
  if (dt > 0.0) {
    clk->t = t + dt;
    clk->steps += 1;
    clk->last_dt = dt;
  }
}

__global__ void zero_kernel(unsigned* p) { *p = 0u; }

// Compensated (Neumaier) float64 accumulation.
struct Acc {
  double s, c;
  __device__ void add(double x) {
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  __device__ double value() const { return s + c; }
};

// The conservation totals (hydro/diagnostics.wgsl channels 0-8, src/sim.ts:1808), per block in
// compensated float64: mass, momentum (3), kinetic, internal (E - KE), total energy, floored
// cells; the Mach maximum separately. Writes NDIAG doubles per block.
constexpr int NDIAG = 9;
__global__ void diag_partial_kernel(const KParams P, const float4* __restrict__ u1, const float4* __restrict__ u2,
                                    size_t ncell, double* __restrict__ part) {
  Acc acc[8];
#pragma unroll
  for (int i = 0; i < 8; i++) acc[i] = Acc{0.0, 0.0};
  double mach = 0.0;
  const double dv = P.dv;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < ncell; o += (size_t)gridDim.x * blockDim.x) {
    const float4 a = __ldg(u1 + o), b = __ldg(u2 + o);
    const double rho = fmax((double)a.x, (double)P.rho_floor);
    const double vx = a.y / rho, vy = a.z / rho, vz = a.w / rho;
    const double v2 = vx * vx + vy * vy + vz * vz;
    const double p = fmax((double)P.gm1 * b.y, (double)P.p_floor);
    const double cs = sqrt((double)P.gamma * p / rho);
    acc[0].add(rho * dv);
    acc[1].add((double)a.y * dv);
    acc[2].add((double)a.z * dv);
    acc[3].add((double)a.w * dv);
    acc[4].add(0.5 * rho * v2 * dv);
    acc[5].add(((double)b.x - 0.5 * rho * v2) * dv);
    acc[6].add((double)b.x * dv);
    acc[7].add((a.x <= P.rho_floor * 1.0001f || p <= P.p_floor * 1.0001) ? 1.0 : 0.0);
    mach = fmax(mach, sqrt(v2) / cs);
  }
  // block reduction in a fixed order: each warp's lanes, then the warps
  __shared__ double sh[32][NDIAG];
  double v[NDIAG];
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = acc[i].value();
  v[8] = mach;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int i = 0; i < NDIAG; i++) {
      const double o = __shfl_down_sync(0xffffffffu, v[i], off);
      v[i] = (i == 8) ? fmax(v[i], o) : v[i] + o;
    }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int i = 0; i < NDIAG; i++) sh[warp][i] = v[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    for (int i = 0; i < NDIAG; i++) {
      Acc s{0.0, 0.0};
      double mx = 0.0;
      for (int w = 0; w < nw; w++) {
        if (i == 8) mx = fmax(mx, sh[w][i]);
        else s.add(sh[w][i]);
      }
      part[(size_t)blockIdx.x * NDIAG + i] = (i == 8) ? mx : s.value();
    }
  }
}

__global__ void diag_final_kernel(const double* __restrict__ part, int nblocks, double* __restrict__ out) {
  const int i = threadIdx.x;
  if (i >= NDIAG) return;
  Acc s{0.0, 0.0};
  double mx = 0.0;
  for (int b = 0; b < nblocks; b++) {
    const double x = part[(size_t)b * NDIAG + i];
    if (i == 8) mx = fmax(mx, x);
    else s.add(x);
  }
  out[i] = (i == 8) ? mx : s.value();
}

// The extended channels (diag_ext.cuh) of a uniform grid: cell centres from the box centre, as
// diagnostics.wgsl:52-56 has them (a 2D grid in the plane z = 0, a 1D one on the x axis).
__global__ void diag_ext_partial_kernel(const KParams P, const float4* __restrict__ u1, const float4* __restrict__ u2,
                                        size_t ncell, double* __restrict__ part) {
  dext::Ext e;
  e.init();
  const int nx = P.n[0], ny = P.n[1], nz = P.n[2];
  const double dx = P.dx, dv = P.dv;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < ncell; o += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(o % nx), j = (int)((o / nx) % ny), k = (int)(o / ((size_t)nx * ny));
    const double x = (i + 0.5 - 0.5 * nx) * dx;
    const double y = ny > 1 ? (j + 0.5 - 0.5 * ny) * dx : 0.0;
    const double z = nz > 1 ? (k + 0.5 - 0.5 * nz) * dx : 0.0;
    e.cell(__ldg(u1 + o), __ldg(u2 + o), P, dv, x, y, z);
  }
  dext::block_reduce(e, part + (size_t)blockIdx.x * dext::N);
}

// ---------------------------------------------------------------------------------------------
// Host launchers.

cudaError_t launch_diag_ext(const KParams& P, const float4* u1, const float4* u2, size_t ncell, double* part, double* out,
                            cudaStream_t s) {
  const int g = diag_blocks(ncell);
  diag_ext_partial_kernel<<<g, 256, 0, s>>>(P, u1, u2, ncell, part);
  dext::final_kernel<<<1, 32, 0, s>>>(part, g, out);
  return cudaGetLastError();
}

template <int DIM, int RECON, bool ISEN>
static cudaError_t launch_sweep_t(const KParams& P, const float4* u1, const float4* u2, float4* o1, float4* o2,
                                  const DevClock* clk, unsigned* rate_out, int tz, const SweepMaps* maps, int* err,
                                  cudaStream_t s) {
  using G = Geo<DIM, RECON>;
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(sweep_kernel<DIM, RECON, ISEN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)G::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    // all of the unified L1/shared storage as shared memory, so that two CTAs fit per SM
    e = cudaFuncSetAttribute(sweep_kernel<DIM, RECON, ISEN>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  dim3 grid((P.n[0] + G::TX - 1) / G::TX, DIM >= 2 ? (P.n[1] + G::TY - 1) / G::TY : 1,
            DIM == 3 ? (P.n[2] + tz - 1) / tz : 1);
  static const CUtensorMap none{};
  const bool tma = DIM == 3 && maps && maps->valid;
  sweep_kernel<DIM, RECON, ISEN><<<grid, G::NT, G::SMEM_BYTES, s>>>(P, u1, u2, o1, o2, clk, rate_out, tz,
                                                                    tma ? maps->u1 : none, tma ? maps->u2 : none,
                                                                    tma ? maps->zofs : 0, tma ? 1 : 0, err);
  return cudaGetLastError();
}

template <int DIM, int RECON>
static cudaError_t launch_sweep_r(const KParams& P, bool isen, const float4* u1, const float4* u2, float4* o1, float4* o2,
                                  const DevClock* clk, unsigned* rate_out, int tz, const SweepMaps* maps, int* err,
                                  cudaStream_t s) {
  if constexpr (RECON == R_PPM) {
    return launch_sweep_t<DIM, RECON, false>(P, u1, u2, o1, o2, clk, rate_out, tz, maps, err, s);
  } else {
    return isen ? launch_sweep_t<DIM, RECON, true>(P, u1, u2, o1, o2, clk, rate_out, tz, maps, err, s)
                : launch_sweep_t<DIM, RECON, false>(P, u1, u2, o1, o2, clk, rate_out, tz, maps, err, s);
  }
}

template <int DIM>
static cudaError_t launch_sweep_d(const KParams& P, int recon, bool isen, const float4* u1, const float4* u2, float4* o1,
                                  float4* o2, const DevClock* clk, unsigned* rate_out, int tz, const SweepMaps* maps,
                                  int* err, cudaStream_t s) {
  switch (recon) {
    case R_MINMOD: return launch_sweep_r<DIM, R_MINMOD>(P, isen, u1, u2, o1, o2, clk, rate_out, tz, maps, err, s);
    case R_MC: return launch_sweep_r<DIM, R_MC>(P, isen, u1, u2, o1, o2, clk, rate_out, tz, maps, err, s);
    case R_VANLEER: return launch_sweep_r<DIM, R_VANLEER>(P, isen, u1, u2, o1, o2, clk, rate_out, tz, maps, err, s);
    case R_KOREN: return launch_sweep_r<DIM, R_KOREN>(P, isen, u1, u2, o1, o2, clk, rate_out, tz, maps, err, s);
    case R_PPM: return launch_sweep_r<DIM, R_PPM>(P, isen, u1, u2, o1, o2, clk, rate_out, tz, maps, err, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int RECON, bool ISEN>
static cudaError_t launch_rows_t(const KParams& P, const float4* u1, const float4* u2, float4* o1, float4* o2,
                                 const DevClock* clk, unsigned* rate_out, int rows, cudaStream_t s) {
  using G = RowGeo<RECON>;
  static_assert(G::SMEM_BYTES <= 48 * 1024, "the row march fits the default shared-memory limit");
  dim3 grid((P.n[0] + G::TX - 1) / G::TX, (P.n[1] + rows - 1) / rows, 1);
  sweep_rows_kernel<RECON, ISEN><<<grid, G::NT, G::SMEM_BYTES, s>>>(P, u1, u2, o1, o2, clk, rate_out, rows);
  return cudaGetLastError();
}

template <int RECON>
static cudaError_t launch_rows_r(const KParams& P, bool isen, const float4* u1, const float4* u2, float4* o1, float4* o2,
                                 const DevClock* clk, unsigned* rate_out, int rows, cudaStream_t s) {
  if constexpr (RECON == R_PPM) {
    return launch_rows_t<RECON, false>(P, u1, u2, o1, o2, clk, rate_out, rows, s);
  } else {
    return isen ? launch_rows_t<RECON, true>(P, u1, u2, o1, o2, clk, rate_out, rows, s)
                : launch_rows_t<RECON, false>(P, u1, u2, o1, o2, clk, rate_out, rows, s);
  }
}

static cudaError_t launch_rows(const KParams& P, int recon, bool isen, const float4* u1, const float4* u2, float4* o1,
                               float4* o2, const DevClock* clk, unsigned* rate_out, int rows, cudaStream_t s) {
  switch (recon) {
    case R_MINMOD: return launch_rows_r<R_MINMOD>(P, isen, u1, u2, o1, o2, clk, rate_out, rows, s);
    case R_MC: return launch_rows_r<R_MC>(P, isen, u1, u2, o1, o2, clk, rate_out, rows, s);
    case R_VANLEER: return launch_rows_r<R_VANLEER>(P, isen, u1, u2, o1, o2, clk, rate_out, rows, s);
    case R_KOREN: return launch_rows_r<R_KOREN>(P, isen, u1, u2, o1, o2, clk, rate_out, rows, s);
    case R_PPM: return launch_rows_r<R_PPM>(P, isen, u1, u2, o1, o2, clk, rate_out, rows, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_sweep(const KParams& P, int ndim, int recon, bool isen, const float4* u1, const float4* u2, float4* o1,
                         float4* o2, const DevClock* clk, unsigned* rate_out, cudaStream_t s, int tz,
                         const SweepMaps* maps, int* err) {
  switch (ndim) {
    case 1: return launch_sweep_d<1>(P, recon, isen, u1, u2, o1, o2, clk, rate_out, 1, nullptr, err, s);
    case 2:
      // tz > 0: the march along y with tz rows a CTA; else the tile form
      return tz > 0 ? launch_rows(P, recon, isen, u1, u2, o1, o2, clk, rate_out, tz, s)
                    : launch_sweep_d<2>(P, recon, isen, u1, u2, o1, o2, clk, rate_out, 1, nullptr, err, s);
    case 3:
      return launch_sweep_d<3>(P, recon, isen, u1, u2, o1, o2, clk, rate_out, tz > 0 ? tz : SWEEP_TZ_DEFAULT, maps,
                               err, s);
    default: return cudaErrorInvalidValue;
  }
}

size_t sweep_smem_bytes(int ndim, int recon) {
  const bool ppm = recon == R_PPM;
  switch (ndim) {
    case 1: return ppm ? Geo<1, R_PPM>::SMEM_BYTES : Geo<1, R_MINMOD>::SMEM_BYTES;
    case 2: return ppm ? Geo<2, R_PPM>::SMEM_BYTES : Geo<2, R_MINMOD>::SMEM_BYTES;
    default: return ppm ? Geo<3, R_PPM>::SMEM_BYTES : Geo<3, R_MINMOD>::SMEM_BYTES;
  }
}

int sweep_min_cells(int recon) { return recon == R_PPM ? 3 : 2; }

cudaError_t launch_rate(const KParams& P, const float4* u1, const float4* u2, size_t ncell, unsigned* out, cudaStream_t s) {
  zero_kernel<<<1, 1, 0, s>>>(out);
  int blocks = (int)((ncell + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (blocks < 1) blocks = 1;
  rate_kernel<<<blocks, 256, 0, s>>>(P, u1, u2, ncell, out);
  return cudaGetLastError();
}

cudaError_t launch_clock(DevClock* clk, unsigned* rates, int slot, cudaStream_t s) {
  clock_kernel<<<1, 1, 0, s>>>(clk, rates, slot);
  return cudaGetLastError();
}

int diag_blocks(size_t ncell) {
  size_t b = (ncell + 255) / 256;
  if (b > 148 * 4) b = 148 * 4;
  return b < 1 ? 1 : (int)b;
}

cudaError_t launch_diag(const KParams& P, const float4* u1, const float4* u2, size_t ncell, double* part, double* out,
                        cudaStream_t s) {
  const int blocks = diag_blocks(ncell);
  diag_partial_kernel<<<blocks, 256, 0, s>>>(P, u1, u2, ncell, part);
  diag_final_kernel<<<1, 32, 0, s>>>(part, blocks, out);
  return cudaGetLastError();
}

// Tensor maps of a 3D state for the sweep's staging: each array as a 3D tensor of floats
// (4 nx, ny, planes), box (4 WX, WY, 1) of the reconstruction's stencil region. `base` is the start
// of the allocation (halo planes included); the sweep adds zofs to a plane's index.
bool encode_sweep_maps(SweepMaps* m, const float4* base1, const float4* base2, int nx, int ny, int planes, int zofs,
                       int recon) {
  m->valid = false;
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                              const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Encode encode = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      fn = nullptr;
    return reinterpret_cast<Encode>(fn);
  }();
  if (!encode) return false;
  const int wx = (recon == R_PPM ? Geo<3, R_PPM>::WX : Geo<3, R_MINMOD>::WX);
  const int wy = (recon == R_PPM ? Geo<3, R_PPM>::WY : Geo<3, R_MINMOD>::WY);
  if (nx < wx || ny < wy) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)4 * nx, (cuuint64_t)ny, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * sizeof(float4), (cuuint64_t)nx * ny * sizeof(float4)};
  const cuuint32_t box[3] = {(cuuint32_t)(4 * wx), (cuuint32_t)wy, 1u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  const float4* bases[2] = {base1, base2};
  CUtensorMap* maps[2] = {&m->u1, &m->u2};
  for (int i = 0; i < 2; i++) {
    if (((uintptr_t)bases[i] & 15u) != 0) return false;
    if (encode(maps[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)bases[i], dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  }
  m->zofs = zofs;
  m->valid = true;
  return true;
}

}  // namespace shz
