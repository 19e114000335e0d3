// ORACLE — test infrastructure only. Nothing in the shipped library links, calls or loads this
// file; only tests/ use it, and only as the checker.
//
// A float64 CPU restatement of one step of the reference's block grid (src/amr), on a block table
// and a state the caller gives, pass by pass as the reference runs them (AmrSim.encodeSteps,
// src/amr/amr_sim.ts:2709-2946):
//   assemble  primitives of every block with two ghost layers (amr/assemble.wgsl:78-154): own
//             cells, restriction of a refined block's children (amr/cons.wgsl:19-43 u_at),
//             prolongation beyond a coarser face (assemble.wgsl:47-75 from_coarse, cons.wgsl:53-125),
//             images beyond the domain's faces (amr/grid.wgsl:186-222 ghost_src); the leaves'
//             signal rate per unit cell size (the dt reduction's first stage);
//   predict   half steps of every leaf and its first ghost layer (amr/predict.wgsl:184-221): at the
//             source for a same-level or boundary ghost, in place with the transverse slopes
//             dropped at the rim for a ghost beyond a coarser face;
//   update    fluxes and the conservative update of every leaf cell (amr/update.wgsl:327-560), a
//             face beside a refined neighbour taking the mean of the fine fluxes through it
//             (update.wgsl:207-295 match_faces, computed as hydro/flux.wgsl:254-347 flux_between);
//   flag      the Löhner indicator per leaf (amr/flag.wgsl:66-155);
//   regrid    the new tree's leaves filled from the old one: copy, prolongation with the kinetic
//             energy kept consistent, restriction (amr/regrid.wgsl:41-139).
// The per-cell arithmetic (limiters, density along the adiabat, Hancock step, HLLC, dual energy)
// is the reference's CPU scheme's, src/reference/hydro.ts, shared with the uniform-grid oracle
// (hydro_ref.h): the block grid's shaders call the same functions as the uniform grid's.
//
// One rule is not the reference's: edge and corner ghosts. The reference leaves them unwritten
// (assemble.wgsl:86, kind 2); a ghost beyond a coarser face at the rim of the face is predicted
// in place and its masked transverse neighbours, edge ghosts, still enter its shock flag and
// positivity check (hydro/predictor.wgsl:110-131), so there the reference reads whatever the
// texture held. This oracle resolves an edge or corner ghost one axis at a time through the table
// (the rule the CUDA path documents for the same texels): across the first out-of-range axis to
// the same-level neighbour or the boundary image, the remaining axes in that block's frame, and
// where a hop meets a coarser block the remaining axes are clamped into the block (the face ghost
// beside it).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "hydro_ref.h"

extern "C" {

typedef struct oamr_params {
  int32_t ndim;         // 2 or 3
  int32_t nr;           // root blocks per side
  int32_t cap;          // block slots
  double dx0;           // level-0 cell size
  double gamma;
  double rho_floor;
  double p_floor;
  double eta_dual;
  double shock_thresh;
  int32_t riemann;      // 0 hllc, 1 hll
  int32_t recon;        // 0 minmod, 1 mc, 2 vanleer, 3 koren
  int32_t isentropic;
  int32_t signal_dims;  // the multiple of the sound speed in the signal rate (hydro.ts:254: 3)
} oamr_params;

}  // extern "C"

namespace {

using namespace oracle;

constexpr int BS = 16, NG = 2, PAD = BS + 2 * NG, PP = BS + 2, BTS = 32, RGS = 12;
const double NaN = std::numeric_limits<double>::quiet_NaN();

struct Cons {
  double a[4];  // rho, mx, my, mz
  double b[4];  // E, e_int, rho s, solid flag
};

// Where the value of a (possibly ghost) cell comes from (amr/grid.wgsl:186-222 Src).
struct Src {
  int kind;  // 0 a cell at the same level, 1 beyond a face whose neighbour is coarser, 2 edge/corner
  int slot;  // kind 0: the block holding the cell; kind 1: the coarser leaf
  int from;  // the block in whose frame l is given
  int l[3];
  double flip[3];
};

struct Amr {
  oamr_params P;
  int nd, CB, WN, PN;
  std::vector<int32_t> bt;
  std::vector<double> U;   // cap x CB x 8: (u1, u2) per cell
  std::vector<double> W;   // cap x WN x 7: rho, vx, vy, vz, p, s, cs per texel
  std::vector<double> PQ;  // cap x PN x 8: half-step rho, v, p, s, shock flag, first-order flag
  int threads = 1;

  explicit Amr(const oamr_params& p) : P(p) {
    nd = p.ndim;
    CB = nd == 3 ? BS * BS * BS : BS * BS;
    WN = nd == 3 ? PAD * PAD * PAD : PAD * PAD;
    PN = nd == 3 ? PP * PP * PP : PP * PP;
    bt.assign((size_t)p.cap * BTS, -1);
    U.assign((size_t)p.cap * CB * 8, 0.0);
    W.assign((size_t)p.cap * WN * 7, NaN);
    PQ.assign((size_t)p.cap * PN * 8, NaN);
  }

  int at(int slot, int i) const { return bt[(size_t)slot * BTS + i]; }
  // amr/grid.wgsl:64-66 blk_leaf: flags (word 4) active and leaf.
  bool leaf(int slot) const { return (at(slot, 4) & 3) == 3; }
  double dx_of(int slot) const { return P.dx0 / std::ldexp(1.0, at(slot, 0)); }

  int cell_ix(const int* l) const { return nd == 3 ? (l[2] * BS + l[1]) * BS + l[0] : l[1] * BS + l[0]; }
  int wtex(const int* l) const {
    return nd == 3 ? ((l[2] + NG) * PAD + (l[1] + NG)) * PAD + (l[0] + NG) : (l[1] + NG) * PAD + (l[0] + NG);
  }
  int ptex(const int* l) const {
    return nd == 3 ? ((l[2] + 1) * PP + (l[1] + 1)) * PP + (l[0] + 1) : (l[1] + 1) * PP + (l[0] + 1);
  }
  double* u_ptr(int slot, const int* l) { return &U[((size_t)slot * CB + cell_ix(l)) * 8]; }
  const double* u_ptr(int slot, const int* l) const { return &U[((size_t)slot * CB + cell_ix(l)) * 8]; }
  const double* w_ptr(int slot, const int* l) const { return &W[((size_t)slot * WN + wtex(l)) * 7]; }
  double* w_ptr(int slot, const int* l) { return &W[((size_t)slot * WN + wtex(l)) * 7]; }
  const double* p_ptr(int slot, const int* l) const { return &PQ[((size_t)slot * PN + ptex(l)) * 8]; }
  double* p_ptr(int slot, const int* l) { return &PQ[((size_t)slot * PN + ptex(l)) * 8]; }

  // amr/grid.wgsl:186-222 ghost_src, with hydro/boundary.wgsl:45-58 bc_ghost_cell / bc_vsign for
  // the domain's faces (1 outflow: the edge cell; 2 reflecting: the mirror image, the normal
  // velocity reversed). Periodic faces have a same-level neighbour in the table.
  Src ghost_src(int slot, const int* l) const {
    Src s;
    s.kind = 0;
    s.slot = slot;
    s.from = slot;
    for (int a = 0; a < 3; a++) { s.l[a] = l[a]; s.flip[a] = 1.0; }
    int out = 0, axis = 0;
    for (int a = 0; a < nd; a++)
      if (l[a] < 0 || l[a] >= BS) { out++; axis = a; }
    if (out == 0) return s;
    if (out > 1) { s.kind = 2; return s; }
    const bool upper = l[axis] >= BS;
    const int nb = at(slot, 6 + 2 * axis + (upper ? 1 : 0));
    if (nb >= 0) {
      s.slot = nb;
      s.l[axis] = l[axis] + (upper ? -BS : BS);
    } else if (nb == -1) {
      s.kind = 1;
      s.slot = at(slot, 20 + 2 * axis + (upper ? 1 : 0));
    } else {
      const int k = -1 - nb;
      if (k == 2) {
        s.l[axis] = upper ? 2 * BS - 1 - l[axis] : -1 - l[axis];
        s.flip[axis] = -1.0;
      } else {
        s.l[axis] = upper ? BS - 1 : 0;
      }
    }
    return s;
  }

  // An edge or corner ghost resolved one axis at a time (the one rule that is not the
  // reference's: see the file's header). A face ghost is ghost_src's.
  Src ghost_src_any(int slot, const int* l) const {
    int cur = slot;
    int m[3] = {l[0], l[1], l[2]};
    double flip[3] = {1, 1, 1};
    for (int hop = 0; hop < nd; hop++) {
      int out = 0, axis = -1;
      for (int a = 0; a < nd; a++)
        if (m[a] < 0 || m[a] >= BS) {
          out++;
          if (axis < 0) axis = a;
        }
      if (out <= 1) break;
      const bool upper = m[axis] >= BS;
      const int nb = at(cur, 6 + 2 * axis + (upper ? 1 : 0));
      if (nb >= 0) {
        cur = nb;
        m[axis] += upper ? -BS : BS;
      } else if (nb <= -2) {
        if (-1 - nb == 2) {
          m[axis] = upper ? 2 * BS - 1 - m[axis] : -1 - m[axis];
          flip[axis] = -flip[axis];
        } else {
          m[axis] = upper ? BS - 1 : 0;
        }
      } else {
        for (int a = 0; a < nd; a++)
          if (a != axis) m[a] = std::min(std::max(m[a], 0), BS - 1);
      }
    }
    Src s = ghost_src(cur, m);
    for (int a = 0; a < 3; a++) s.flip[a] *= flip[a];
    return s;
  }

  // amr/cons.wgsl:19-43 u_at: a leaf's own cell, or the mean of the 2^ndim cells of the leaf
  // child under it; the placeholder state where the child is refined further (2:1 balance keeps
  // every leaf's stencil away from there).
  Cons u_at(int slot, const int* l) const {
    Cons u;
    if (leaf(slot)) {
      const double* p = u_ptr(slot, l);
      for (int i = 0; i < 4; i++) { u.a[i] = p[i]; u.b[i] = p[4 + i]; }
      return u;
    }
    const int h[3] = {l[0] >= BS / 2, l[1] >= BS / 2, nd == 3 ? (l[2] >= BS / 2) : 0};
    const int ch = at(slot, 12 + (h[0] | (h[1] << 1) | (h[2] << 2)));
    if (ch < 0 || !leaf(ch)) {
      const double a0[4] = {1, 0, 0, 0}, b0[4] = {1, 1, 0, 0};
      for (int i = 0; i < 4; i++) { u.a[i] = a0[i]; u.b[i] = b0[i]; }
      return u;
    }
    for (int i = 0; i < 4; i++) { u.a[i] = 0; u.b[i] = 0; }
    const int nz = nd == 3 ? 2 : 1;
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < 2; j++)
        for (int i = 0; i < 2; i++) {
          const int f[3] = {2 * (l[0] - (BS / 2) * h[0]) + i, 2 * (l[1] - (BS / 2) * h[1]) + j,
                            nd == 3 ? 2 * (l[2] - (BS / 2) * h[2]) + k : 0};
          const double* p = u_ptr(ch, f);
          for (int q = 0; q < 4; q++) { u.a[q] += p[q]; u.b[q] += p[4 + q]; }
        }
    const double w = nd == 3 ? 0.125 : 0.25;
    for (int q = 0; q < 4; q++) { u.a[q] *= w; u.b[q] *= w; }
    return u;
  }

  // amr/cons.wgsl:48-51 u_near: a kind-0 cell with the boundary's velocity signs; false otherwise.
  bool u_near(int slot, const int* l, Cons& u) const {
    const Src s = ghost_src(slot, l);
    if (s.kind != 0) return false;
    u = u_at(s.slot, s.l);
    for (int a = 0; a < 3; a++) u.a[1 + a] *= s.flip[a];
    return true;
  }

  // The prolongation's single slope (the limiter's limit4: MC for Koren, limiters/koren.wgsl:57).
  double lim4(double a, double b) const { return limiter(P.recon == KOREN ? MC : P.recon, a, b, 0.0); }

  // amr/cons.wgsl:53-70 mom_slope / slope_between: limited slopes, the momentum's by the product
  // rule from the density's and the velocity's.
  Cons slope_between(const Cons& c, const Cons& m, const Cons& p) const {
    Cons s;
    s.a[0] = lim4(c.a[0] - m.a[0], p.a[0] - c.a[0]);
    const double ic = 1 / std::max(c.a[0], P.rho_floor), im = 1 / std::max(m.a[0], P.rho_floor),
                 ip = 1 / std::max(p.a[0], P.rho_floor);
    for (int i = 0; i < 3; i++) {
      const double vc = c.a[1 + i] * ic, vm = m.a[1 + i] * im, vp = p.a[1 + i] * ip;
      s.a[1 + i] = vc * s.a[0] + c.a[0] * lim4(vc - vm, vp - vc);
    }
    for (int i = 0; i < 4; i++) s.b[i] = lim4(c.b[i] - m.b[i], p.b[i] - c.b[i]);
    return s;
  }

  struct Slopes {
    Cons s[3];
    double f;
  };

  // amr/cons.wgsl:78-106 prolong_slopes: per-axis slopes scaled back by one common factor.
  Slopes prolong_slopes(const Cons& uc, const Cons* m, const bool* mok, const Cons* p, const bool* pok) const {
    Slopes sl;
    double drop[3] = {0, 0, 0};
    for (int a = 0; a < 3; a++) {
      for (int i = 0; i < 4; i++) { sl.s[a].a[i] = 0; sl.s[a].b[i] = 0; }
      if (a < nd && mok[a] && pok[a]) sl.s[a] = slope_between(uc, m[a], p[a]);
      drop[0] += std::fabs(sl.s[a].a[0]);
      drop[1] += std::fabs(sl.s[a].b[0]);
      drop[2] += std::fabs(sl.s[a].b[1]);
    }
    const double room[3] = {0.5 * std::max(uc.a[0], 0.0), 0.5 * std::max(uc.b[0], 0.0), 0.5 * std::max(uc.b[1], 0.0)};
    double f = 1;
    for (int i = 0; i < 3; i++) f = std::min(f, std::min(1.0, room[i] / std::max(0.25 * drop[i], 1e-37)));
    sl.f = f;
    return sl;
  }
  // amr/cons.wgsl:109-123 prolong_child.
  static Cons prolong_child(const Cons& uc, const Slopes& s, const int* par) {
    double off[3];
    for (int a = 0; a < 3; a++) off[a] = s.f * (par[a] - 0.5) * 0.5;
    Cons u;
    for (int i = 0; i < 4; i++) {
      u.a[i] = uc.a[i] + off[0] * s.s[0].a[i] + off[1] * s.s[1].a[i] + off[2] * s.s[2].a[i];
      u.b[i] = uc.b[i] + off[0] * s.s[0].b[i] + off[1] * s.s[1].b[i] + off[2] * s.s[2].b[i];
    }
    return u;
  }

  // amr/assemble.wgsl:47-75 from_coarse: fine ghost l of block `from`, prolonged from the coarser
  // leaf cs beyond the face, its slopes from cs's neighbours.
  Cons from_coarse(int from, const int* l, int cs) const {
    const int nc = (P.nr * BS) << at(cs, 0);
    int lc[3], par[3];
    for (int a = 0; a < 3; a++) {
      const int gf = a < nd ? at(from, 1 + a) * BS + l[a] : 0;
      int gc = gf >> 1;  // floor(gf / 2)
      gc = ((gc % nc) + nc) % nc;
      lc[a] = a < nd ? gc - at(cs, 1 + a) * BS : 0;
      par[a] = a < nd ? (gf & 1) : 0;
    }
    Cons uc, m[3], p[3];
    bool mok[3] = {false, false, false}, pok[3] = {false, false, false};
    if (!u_near(cs, lc, uc)) {
      const double a0[4] = {1, 0, 0, 0}, b0[4] = {1, 1, 0, 0};
      for (int i = 0; i < 4; i++) { uc.a[i] = a0[i]; uc.b[i] = b0[i]; }
    }
    for (int a = 0; a < nd; a++) {
      int q[3] = {lc[0], lc[1], lc[2]};
      q[a] -= 1;
      mok[a] = u_near(cs, q, m[a]);
      q[a] += 2;
      pok[a] = u_near(cs, q, p[a]);
    }
    return prolong_child(uc, prolong_slopes(uc, m, mok, p, pok), par);
  }

  // hydro/prim.wgsl:26-51 (hydro.ts:233-257 primitives): (rho, v, p, s, cs).
  void prim(const Cons& u, double* w) const {
    const double rho = std::max(u.a[0], P.rho_floor);
    double p = (P.gamma - 1) * u.b[1];
    if (!(p >= P.p_floor)) p = P.p_floor;
    w[0] = rho;
    w[1] = u.a[1] / rho;
    w[2] = u.a[2] / rho;
    w[3] = u.a[3] / rho;
    w[4] = p;
    w[5] = u.b[2] / rho;
    w[6] = std::sqrt(P.gamma * p / rho);
  }

  // assemble.wgsl:78-154 for one block: every texel of its 20^ndim region from its source. Returns
  // the largest signal rate per unit cell size over a leaf's own cells (0 for a parent).
  double assemble_block(int slot) {
    double rmax = 0;
    const double inv_dx = 1 / dx_of(slot);
    const int zlo = nd == 3 ? -NG : 0, zhi = nd == 3 ? BS + NG : 1;
    for (int z = zlo; z < zhi; z++)
      for (int y = -NG; y < BS + NG; y++)
        for (int x = -NG; x < BS + NG; x++) {
          const int l[3] = {x, y, z};
          const bool inside = x >= 0 && x < BS && y >= 0 && y < BS && (nd == 2 || (z >= 0 && z < BS));
          Cons u;
          if (inside) {
            u = u_at(slot, l);
          } else {
            const Src s = ghost_src_any(slot, l);
            if (s.kind == 0) u = u_at(s.slot, s.l);
            else if (s.kind == 1) u = from_coarse(s.from, s.l, s.slot);
            else continue;  // unresolved: left NaN (never met on a 2:1-balanced mesh)
            for (int a = 0; a < 3; a++) u.a[1 + a] *= s.flip[a];
          }
          double* w = w_ptr(slot, l);
          prim(u, w);
          if (inside && leaf(slot)) {
            const double r = std::fabs(w[1]) + std::fabs(w[2]) + std::fabs(w[3]) + P.signal_dims * w[6];
            rmax = std::max(rmax, r * inv_dx);
          }
        }
    return rmax;
  }

  // hydro.ts:268-293: the edge increments of cell c along one axis from its neighbours m and p
  // (limited slopes, or Koren's increments per face; the density along the adiabat, :260-265).
  void edges(const double* m, const double* c, const double* p, double* su, double* sd) const {
    const double sc[NQ] = {c[0], c[6], c[6], c[6], c[4], 0.0};
    for (int v = 0; v < NQ; v++) su[v] = limiter(P.recon, c[v] - m[v], p[v] - c[v], sc[v]);
    for (int v = 0; v < NQ; v++) sd[v] = limiter(P.recon, p[v] - c[v], c[v] - m[v], sc[v]);
    if (P.isentropic) {
      double inc, b;
      isen_inc(m, c, p, su[4], true, P.recon, P.gamma, &inc, &b);
      su[0] += std::min(std::max(inc - su[0], -b), b);
      isen_inc(m, c, p, sd[4], false, P.recon, P.gamma, &inc, &b);
      sd[0] += std::min(std::max(inc - sd[0], -b), b);
    }
  }

  // amr/predict.wgsl:184-221 over one leaf: its cells and first ghost layer, with
  // hydro/predictor.wgsl:46-209 (hydro.ts:272-322 predictRaw) and the mask of the rim ghosts.
  void predict_block(int slot, double dt) {
    const double h = 0.5 * dt / dx_of(slot);
    const int zlo = nd == 3 ? -1 : 0, zhi = nd == 3 ? BS + 1 : 1;
    for (int z = zlo; z < zhi; z++)
      for (int y = -1; y < BS + 1; y++)
        for (int x = -1; x < BS + 1; x++) {
          const int l[3] = {x, y, z};
          const Src s = ghost_src(slot, l);
          double* out = p_ptr(slot, l);
          if (s.kind == 2) continue;
          const bool at_source = s.kind == 0;
          const int src = at_source ? s.slot : slot;
          const int c0[3] = {at_source ? s.l[0] : l[0], at_source ? s.l[1] : l[1], at_source ? s.l[2] : l[2]};
          double mask[3] = {1, 1, 1};
          if (!at_source)
            for (int a = 0; a < nd; a++) mask[a] = (l[a] == 0 || l[a] == BS - 1) ? 0.0 : 1.0;
          const double* c = w_ptr(src, c0);
          double su[3][NQ] = {}, sd[3][NQ] = {};
          double conv = 0, jump = -std::numeric_limits<double>::infinity();
          for (int a = 0; a < nd; a++) {
            int lm[3] = {c0[0], c0[1], c0[2]}, lp[3] = {c0[0], c0[1], c0[2]};
            lm[a] -= 1;
            lp[a] += 1;
            const double* m = w_ptr(src, lm);
            const double* p = w_ptr(src, lp);
            edges(m, c, p, su[a], sd[a]);
            conv += p[1 + a] - m[1 + a];
            jump = std::max(jump, std::fabs(p[4] - m[4]) / std::min(p[4], m[4]));
          }
          // hydro/predictor.wgsl:80-131: positivity sees every increment; the half step only
          // the unmasked axes'.
          double big = 0, fall = 0, dv = 0, adv[NQ] = {0, 0, 0, 0, 0, 0}, gradp[3] = {0, 0, 0};
          for (int a = 0; a < nd; a++) {
            big = std::max(big, std::max(std::fabs(su[a][4]), std::fabs(sd[a][4])));
            fall = std::min(fall, std::min(0.5 * su[a][0], -0.5 * sd[a][0]));
            const double k = 0.5 * mask[a];
            for (int v = 0; v < NQ; v++) adv[v] += c[1 + a] * (k * (su[a][v] + sd[a][v]));
            dv += k * (su[a][1 + a] + sd[a][1 + a]);
            gradp[a] = k * (su[a][4] + sd[a][4]);
          }
          const double flag = (conv < 0 && jump > P.shock_thresh) ? 1.0 : 0.0;
          const double rho = c[0], cs = c[6];
          double qh[NQ];
          qh[0] = rho - h * (adv[0] + rho * dv);
          for (int d = 0; d < 3; d++) qh[1 + d] = c[1 + d] - h * (adv[1 + d] + gradp[d] / rho);
          qh[4] = c[4] - h * (adv[4] + rho * cs * cs * dv);
          qh[5] = c[5] - h * adv[5];
          const bool fo = !(qh[0] + fall > 0 && qh[4] - 0.5 * big > 0);
          for (int v = 0; v < NQ; v++) out[v] = fo ? c[v] : qh[v];
          if (at_source)
            for (int a = 0; a < 3; a++) out[1 + a] *= s.flip[a];
          out[6] = flag;
          out[7] = fo ? 1.0 : 0.0;
        }
  }

  // hydro/flux.wgsl:254-347 flux_between (face states as hydro.ts:360-375 side; riemannFlux):
  // the flux through the face between cells a and a + e_axis of block `slot`, lab frame:
  // (m, mx, my, mz, e, ei, s, vn).
  void face_flux(int slot, const int* a, int axis, double* F) const {
    int am[3] = {a[0], a[1], a[2]}, b[3] = {a[0], a[1], a[2]}, bp[3] = {a[0], a[1], a[2]};
    am[axis] -= 1;
    b[axis] += 1;
    bp[axis] += 2;
    double su[NQ], sd[NQ], tu[NQ], td[NQ];
    edges(w_ptr(slot, am), w_ptr(slot, a), w_ptr(slot, b), su, sd);
    edges(w_ptr(slot, a), w_ptr(slot, b), w_ptr(slot, bp), tu, td);
    const double* pa = p_ptr(slot, a);
    const double* pb = p_ptr(slot, b);
    auto side = [&](const double* pr, const double* inc, double sg) {
      const double k = pr[7] != 0 ? 0.0 : 0.5 * sg;
      double f[NQ];
      for (int v = 0; v < NQ; v++) f[v] = pr[v] + k * inc[v];
      Side s;
      s.rho = std::max(f[0], P.rho_floor);
      s.p = std::max(f[4], P.p_floor);
      s.v[0] = f[1 + axis];
      s.v[1] = f[1 + (axis + 1) % 3];
      s.v[2] = f[1 + (axis + 2) % 3];
      s.s = f[5];
      s.cs = std::sqrt(P.gamma * s.p / s.rho);
      s.eint = s.p / (P.gamma - 1);
      return s;
    };
    const Side L = side(pa, su, 1.0), R = side(pb, td, -1.0);
    const Flux f = riemann_flux(L, R, std::max(pa[6], pb[6]), P.riemann == 1);
    F[0] = f.m;
    for (int d = 0; d < 3; d++) F[1 + (axis + d) % 3] = f.mom[d];
    F[4] = f.e;
    F[5] = f.ei;
    F[6] = f.s;
    F[7] = f.vn;
  }

  // amr/update.wgsl:207-295 match_faces (one timestep for every block): where the same-level
  // neighbour beyond face (axis, hi) of cell l is refined, the mean of the fine fluxes through
  // the face as the fine leaf computes them. False where the face keeps its own flux.
  bool match_face(int slot, const int* l, int axis, bool hi, double* F) const {
    const int np = at(slot, 6 + 2 * axis + (hi ? 1 : 0));
    if (np < 0 || leaf(np)) return false;
    const bool upper = !hi;
    const int h[3] = {l[0] >= BS / 2, l[1] >= BS / 2, nd == 3 ? (l[2] >= BS / 2) : 0};
    int bits[3] = {h[0], h[1], h[2]};
    bits[axis] = upper ? 1 : 0;
    if (nd == 2) bits[2] = 0;
    const int ch = at(np, 12 + (bits[0] | (bits[1] << 1) | (bits[2] << 2)));
    if (ch < 0) return false;
    int a0[3] = {2 * (l[0] - (BS / 2) * h[0]), 2 * (l[1] - (BS / 2) * h[1]), nd == 3 ? 2 * (l[2] - (BS / 2) * h[2]) : 0};
    a0[axis] = upper ? BS - 1 : -1;
    const int t1 = (axis + 1) % 3, t2 = (axis + 2) % 3;
    const int n1 = (nd == 2 && t1 == 2) ? 1 : 2, n2 = (nd == 2 && t2 == 2) ? 1 : 2;
    double sum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = 0; j < n2; j++)
      for (int i = 0; i < n1; i++) {
        int a[3] = {a0[0], a0[1], a0[2]};
        a[t1] += i;
        a[t2] += j;
        double f[8];
        face_flux(ch, a, axis, f);
        for (int v = 0; v < 8; v++) sum[v] += f[v];
      }
    const double w = 1.0 / (n1 * n2);
    for (int v = 0; v < 8; v++) F[v] = sum[v] * w;
    return true;
  }

  // amr/update.wgsl:327-560 for one leaf (no gravity, sources or solids): the cell's fluxes, the
  // matched ones at the block's faces, and hydro.ts:430-446 (the update, dual energy, floors).
  void update_block(int slot, double dt, double* out) const {
    const double dtdx = dt / dx_of(slot);
    const int nz = nd == 3 ? BS : 1;
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < BS; y++)
        for (int x = 0; x < BS; x++) {
          const int l[3] = {x, y, z};
          double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
          for (int axis = 0; axis < nd; axis++) {
            double lo[8], hi[8];
            int am[3] = {x, y, z};
            am[axis] -= 1;
            face_flux(slot, am, axis, lo);
            if (l[axis] == 0) match_face(slot, l, axis, false, lo);
            face_flux(slot, l, axis, hi);
            if (l[axis] == BS - 1) match_face(slot, l, axis, true, hi);
            for (int v = 0; v < 8; v++) acc[v] += lo[v] - hi[v];
          }
          const double* u = u_ptr(slot, l);
          const double ph = p_ptr(slot, l)[4];
          const double g = P.gamma;
          const double rho = std::max(u[0] + dtdx * acc[0], P.rho_floor);
          double mom[3];
          for (int d = 0; d < 3; d++) mom[d] = u[1 + d] + dtdx * acc[1 + d];
          double E = u[4] + dtdx * acc[4];
          double eint = u[5] + dtdx * (acc[5] + std::max(ph, P.p_floor) * acc[7]);
          const double ke = (0.5 * (mom[0] * mom[0] + mom[1] * mom[1] + mom[2] * mom[2])) / rho;
          const double eth = E - ke;
          const double emin = P.p_floor / (g - 1);
          if (eth > P.eta_dual * E && eth >= emin) {
            eint = eth;
          } else {
            if (!(eint >= emin)) eint = emin;
            E = ke + eint;
          }
          double* o = out + (size_t)cell_ix(l) * 8;
          o[0] = rho;
          o[1] = mom[0];
          o[2] = mom[1];
          o[3] = mom[2];
          o[4] = E;
          o[5] = eint;
          o[6] = u[6] + dtdx * acc[6];
          o[7] = u[7];
        }
  }

  // amr/flag.wgsl:66-155 over one leaf's cells (gas only): the largest Löhner indicator of density
  // or pressure (EPS 0.01), at least GAS_MIN.
  double flag_block(int slot) const {
    const double EPS = 0.01;
    double mx = 0;
    const int nz = nd == 3 ? BS : 1;
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < BS; y++)
        for (int x = 0; x < BS; x++) {
          const int l[3] = {x, y, z};
          const double* c = w_ptr(slot, l);
          const double r0 = c[0], p0 = c[4];
          double nr = 0, dr = 0, np = 0, dp = 0;
          for (int a = 0; a < nd; a++) {
            int lp[3] = {x, y, z}, lm[3] = {x, y, z};
            lp[a] += 1;
            lm[a] -= 1;
            const double rp = w_ptr(slot, lp)[0], rm = w_ptr(slot, lm)[0];
            const double pp = w_ptr(slot, lp)[4], pm = w_ptr(slot, lm)[4];
            const double sr = rp - 2 * r0 + rm, sp = pp - 2 * p0 + pm;
            const double er = std::fabs(rp - r0) + std::fabs(r0 - rm) + EPS * (std::fabs(rp) + 2 * std::fabs(r0) + std::fabs(rm));
            const double ep = std::fabs(pp - p0) + std::fabs(p0 - pm) + EPS * (std::fabs(pp) + 2 * std::fabs(p0) + std::fabs(pm));
            nr += sr * sr;
            dr += er * er;
            np += sp * sp;
            dp += ep * ep;
          }
          mx = std::max(mx, std::max(std::sqrt(nr / std::max(dr, 1e-30)), std::sqrt(np / std::max(dp, 1e-30))));
        }
    return std::max(mx, 1e-30);
  }

  // amr/regrid.wgsl:41-139 for one leaf of the new tree (row `rg` of the regrid table: kind,
  // source slot, octant, children), from the old state and the old primitives (this object's U
  // and W, assembled from the old tree). Writes 16^ndim cells x 8 into out.
  void regrid_block(const int* rg, double* out) const {
    const int kind = rg[0], src = rg[1], oct = rg[2];
    const int nz = nd == 3 ? BS : 1;
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < BS; y++)
        for (int x = 0; x < BS; x++) {
          const int l[3] = {x, y, z};
          Cons u;
          if (kind == 2) {
            const int lc[3] = {(x >> 1) + (BS / 2) * (oct & 1), (y >> 1) + (BS / 2) * ((oct >> 1) & 1),
                               nd == 3 ? (z >> 1) + (BS / 2) * ((oct >> 2) & 1) : 0};
            Cons uc;
            const double* p = u_ptr(src, lc);
            for (int i = 0; i < 4; i++) { uc.a[i] = p[i]; uc.b[i] = p[4 + i]; }
            Cons m[3], pp[3];
            bool ok[3] = {true, true, true};
            // regrid.wgsl:31-37 cons_from_w: the neighbours' conserved state from the stored
            // primitives (ideal gas: e_int = p / (gamma - 1), as the primitives formed p).
            auto from_w = [&](const int* q) {
              const double* w = w_ptr(src, q);
              Cons c;
              const double rho = std::fabs(w[0]);
              const double eint = w[4] / (P.gamma - 1);
              c.a[0] = rho;
              for (int i = 0; i < 3; i++) c.a[1 + i] = rho * w[1 + i];
              c.b[0] = eint + 0.5 * (c.a[1] * w[1] + c.a[2] * w[2] + c.a[3] * w[3]);
              c.b[1] = eint;
              c.b[2] = rho * w[5];
              c.b[3] = 0;
              return c;
            };
            for (int a = 0; a < nd; a++) {
              int q[3] = {lc[0], lc[1], lc[2]};
              q[a] -= 1;
              m[a] = from_w(q);
              q[a] += 2;
              pp[a] = from_w(q);
            }
            const Slopes sl = prolong_slopes(uc, m, ok, pp, ok);
            const int par[3] = {x & 1, y & 1, nd == 3 ? (z & 1) : 0};
            u = prolong_child(uc, sl, par);
            // regrid.wgsl:75-97: each child's own kinetic energy and its interpolated internal
            // energy, plus one offset that keeps the children's mean total energy the coarse cell's.
            double ke = 0;
            for (int kz = 0; kz < (nd == 3 ? 2 : 1); kz++)
              for (int jy = 0; jy < 2; jy++)
                for (int ix = 0; ix < 2; ix++) {
                  const int pc[3] = {ix, jy, kz};
                  const Cons c = prolong_child(uc, sl, pc);
                  ke += 0.5 * (c.a[1] * c.a[1] + c.a[2] * c.a[2] + c.a[3] * c.a[3]) / std::max(c.a[0], P.rho_floor);
                }
            ke *= nd == 3 ? 0.125 : 0.25;
            u.b[0] = 0.5 * (u.a[1] * u.a[1] + u.a[2] * u.a[2] + u.a[3] * u.a[3]) / std::max(u.a[0], P.rho_floor) +
                     u.b[1] + (uc.b[0] - uc.b[1] - ke);
          } else if (kind == 3) {
            const int h[3] = {x >= BS / 2, y >= BS / 2, nd == 3 ? (z >= BS / 2) : 0};
            const int ch = rg[4 + (h[0] | (h[1] << 1) | (h[2] << 2))];
            for (int i = 0; i < 4; i++) { u.a[i] = 0; u.b[i] = 0; }
            for (int kz = 0; kz < (nd == 3 ? 2 : 1); kz++)
              for (int jy = 0; jy < 2; jy++)
                for (int ix = 0; ix < 2; ix++) {
                  const int f[3] = {2 * (x - (BS / 2) * h[0]) + ix, 2 * (y - (BS / 2) * h[1]) + jy,
                                    nd == 3 ? 2 * (z - (BS / 2) * h[2]) + kz : 0};
                  const double* p = u_ptr(ch, f);
                  for (int i = 0; i < 4; i++) { u.a[i] += p[i]; u.b[i] += p[4 + i]; }
                }
            const double w = nd == 3 ? 0.125 : 0.25;
            for (int i = 0; i < 4; i++) { u.a[i] *= w; u.b[i] *= w; }
          } else {
            const double* p = u_ptr(src, l);
            for (int i = 0; i < 4; i++) { u.a[i] = p[i]; u.b[i] = p[4 + i]; }
          }
          double* o = out + (size_t)cell_ix(l) * 8;
          for (int i = 0; i < 4; i++) { o[i] = u.a[i]; o[4 + i] = u.b[i]; }
        }
  }
};

}  // namespace

extern "C" {

void* oamr_create(const oamr_params* p) {
  if (!p || (p->ndim != 2 && p->ndim != 3) || p->cap < 1 || p->nr < 1) return nullptr;
  return new Amr(*p);
}
void oamr_destroy(void* h) { delete static_cast<Amr*>(h); }
void oamr_set_threads(void* h, int n) { static_cast<Amr*>(h)->threads = n < 1 ? 1 : n; }

// The block table (cap x 32 ints, the reference's BlockTree.table layout, src/amr/tree.ts:652-679).
void oamr_set_table(void* h, const int32_t* table) {
  Amr* a = static_cast<Amr*>(h);
  std::memcpy(a->bt.data(), table, sizeof(int32_t) * a->bt.size());
}

// The state of n blocks: slot[i]'s 16^ndim cells as float32 u1 and u2 (float4 each, x fastest).
void oamr_set_state(void* h, int32_t n, const int32_t* slots, const float* u1, const float* u2) {
  Amr* a = static_cast<Amr*>(h);
  for (int i = 0; i < n; i++)
    for (int c = 0; c < a->CB; c++) {
      double* o = &a->U[((size_t)slots[i] * a->CB + c) * 8];
      const size_t k = ((size_t)i * a->CB + c) * 4;
      for (int q = 0; q < 4; q++) { o[q] = u1[k + q]; o[4 + q] = u2[k + q]; }
    }
}
// The float64 state of n blocks, 16^ndim cells x 8 doubles each.
void oamr_get_state(void* h, int32_t n, const int32_t* slots, double* out) {
  Amr* a = static_cast<Amr*>(h);
  for (int i = 0; i < n; i++)
    std::memcpy(out + (size_t)i * a->CB * 8, &a->U[(size_t)slots[i] * a->CB * 8], sizeof(double) * a->CB * 8);
}

// The assemble over the n blocks of `list` (every block: parents' regions are read by predictions
// at the source). Returns the largest rate per unit cell size over the listed leaves.
double oamr_assemble(void* h, int32_t n, const int32_t* list) {
  Amr* a = static_cast<Amr*>(h);
  std::fill(a->W.begin(), a->W.end(), NaN);
  double r = 0;
#pragma omp parallel for reduction(max : r) num_threads(a->threads) schedule(dynamic)
  for (int i = 0; i < n; i++) r = std::max(r, a->assemble_block(list[i]));
  return r;
}
// One block's primitive region: 20^ndim texels x 7 (rho, vx, vy, vz, p, s, cs), x fastest; NaN
// where nothing was written.
void oamr_get_prims(void* h, int32_t slot, double* out) {
  Amr* a = static_cast<Amr*>(h);
  std::memcpy(out, &a->W[(size_t)slot * a->WN * 7], sizeof(double) * a->WN * 7);
}

// The predict and update passes of one step of dt over the n leaves of `list` (after
// oamr_assemble of the same state); the leaves' state becomes the new one.
void oamr_step(void* h, int32_t n, const int32_t* leaves, double dt) {
  Amr* a = static_cast<Amr*>(h);
  std::fill(a->PQ.begin(), a->PQ.end(), NaN);
#pragma omp parallel for num_threads(a->threads) schedule(dynamic)
  for (int i = 0; i < n; i++) a->predict_block(leaves[i], dt);
  std::vector<double> next((size_t)n * a->CB * 8);
#pragma omp parallel for num_threads(a->threads) schedule(dynamic)
  for (int i = 0; i < n; i++) a->update_block(leaves[i], dt, next.data() + (size_t)i * a->CB * 8);
  for (int i = 0; i < n; i++)
    std::memcpy(&a->U[(size_t)leaves[i] * a->CB * 8], next.data() + (size_t)i * a->CB * 8, sizeof(double) * a->CB * 8);
}
// One leaf's half steps over its cells and first ghost layer: 18^ndim texels x 8 (rho, v, p, s,
// shock flag, first-order flag), x fastest; NaN for edge and corner texels.
void oamr_get_halfsteps(void* h, int32_t slot, double* out) {
  Amr* a = static_cast<Amr*>(h);
  std::memcpy(out, &a->PQ[(size_t)slot * a->PN * 8], sizeof(double) * a->PN * 8);
}

// The Löhner indicators of the n leaves of `list` (after oamr_assemble), one per leaf.
void oamr_flags(void* h, int32_t n, const int32_t* list, double* out) {
  Amr* a = static_cast<Amr*>(h);
#pragma omp parallel for num_threads(a->threads) schedule(dynamic)
  for (int i = 0; i < n; i++) out[i] = a->flag_block(list[i]);
}

// Re-mesh: the new tree's n leaves (slots of the new table) filled from the old state and the old
// primitives (oamr_assemble of the old tree first), by the regrid table's rows (cap x 12 ints,
// BlockTree.regridTable, src/amr/tree.ts:681-693); then the new table replaces the old.
void oamr_regrid(void* h, const int32_t* new_table, const int32_t* rg, int32_t n, const int32_t* leaves) {
  Amr* a = static_cast<Amr*>(h);
  std::vector<double> next((size_t)n * a->CB * 8);
#pragma omp parallel for num_threads(a->threads) schedule(dynamic)
  for (int i = 0; i < n; i++) a->regrid_block(rg + (size_t)leaves[i] * RGS, next.data() + (size_t)i * a->CB * 8);
  for (int i = 0; i < n; i++)
    std::memcpy(&a->U[(size_t)leaves[i] * a->CB * 8], next.data() + (size_t)i * a->CB * 8, sizeof(double) * a->CB * 8);
  std::memcpy(a->bt.data(), new_table, sizeof(int32_t) * a->bt.size());
}

}  // extern "C"
