// C ABI of the host block tree (amr_tree.h): the shz_tree_* entry points.
#include <array>
#include <cstring>
#include <exception>
#include <mutex>
#include <string>

#include "../../include/shaderous_b200.h"
#include "amr_tree.h"

using shz::amr::Block;
using shz::amr::BlockTree;
using shz::amr::RegridOp;

struct shz_tree {
  BlockTree* t;
};

namespace {
std::mutex g_mu;
std::string g_err;
int fail(const char* what) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_err = what;
  return SHZ_E_CONFIG;
}
void emit(const std::vector<RegridOp>& ops, int cap, int32_t* regrid, int32_t* changed) {
  if (changed) *changed = ops.empty() ? 0 : 1;
  if (regrid) {
    if (ops.empty()) std::memset(regrid, 0, sizeof(int32_t) * (size_t)cap * shz::amr::RG_STRIDE);
    else BlockTree::regrid_table(ops, cap, regrid);
  }
}
}  // namespace

extern "C" {

const char* shz_tree_error(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  return g_err.c_str();
}

int shz_tree_create(int32_t ndim, int32_t nr, int32_t max_level, int32_t cap, const int32_t bc_lo[3],
                    const int32_t bc_hi[3], int32_t edge_balance, shz_tree** out) {
  if (!out || !bc_lo || !bc_hi) return fail("shz_tree_create: null argument");
  if (ndim < 1 || ndim > 3 || nr < 1 || max_level < 0 || max_level > shz::amr::MAX_LEVELS || cap < 1)
    return fail("shz_tree_create: ndim 1..3, nr >= 1, max_level 0..7, cap >= 1");
  try {
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) { lo[a] = bc_lo[a]; hi[a] = bc_hi[a]; }
    *out = new shz_tree{new BlockTree(ndim, nr, max_level, cap, lo, hi, edge_balance != 0)};
  } catch (const std::exception& e) {
    return fail(e.what());
  }
  return SHZ_OK;
}

void shz_tree_destroy(shz_tree* t) {
  if (!t) return;
  delete t->t;
  delete t;
}

int shz_tree_adapt(shz_tree* t, const double* ind, double hi, double lo, int32_t* regrid, int32_t* changed) {
  if (!t || !ind) return fail("shz_tree_adapt: null argument");
  try {
    const auto ops = t->t->adapt([&](const Block* b) { return ind[b->slot]; }, hi, lo);
    emit(ops, t->t->cap, regrid, changed);
  } catch (const std::exception& e) {
    return fail(e.what());
  }
  return SHZ_OK;
}

int shz_tree_last_steps(const shz_tree* t, int32_t* out, int32_t max_ints, int32_t* n_ints) {
  if (!t || !n_ints) return fail("shz_tree_last_steps: null argument");
  int32_t n = 0;
  for (const auto& s : t->t->last_steps)
    for (int v : s) {
      if (out && n < max_ints) out[n] = v;
      n++;
    }
  *n_ints = n;
  return n <= max_ints || !out ? SHZ_OK : fail("shz_tree_last_steps: buffer too small");
}

int shz_tree_replay(shz_tree* t, const int32_t* steps, int32_t n_ints, int32_t* regrid, int32_t* changed) {
  if (!t || (!steps && n_ints)) return fail("shz_tree_replay: null argument");
  const int w = 2 + t->t->ndim;
  if (n_ints % w) return fail("shz_tree_replay: steps are [what, level, c...] of 2 + ndim ints");
  std::vector<std::vector<int>> s;
  for (int i = 0; i < n_ints; i += w) s.emplace_back(steps + i, steps + i + w);
  try {
    const auto ops = t->t->replay_adapt(s);
    emit(ops, t->t->cap, regrid, changed);
  } catch (const std::exception& e) {
    return fail(e.what());
  }
  return SHZ_OK;
}

int shz_tree_refine(shz_tree* t, int32_t level, const int32_t c[3], int32_t* n_split) {
  if (!t || !c || !n_split) return fail("shz_tree_refine: null argument");
  const int cc[3] = {c[0], c[1], c[2]};
  Block* b = t->t->get(level, cc);
  if (!b) return fail("shz_tree_refine: no such block");
  try {
    *n_split = (int32_t)t->t->refine(b).size();
  } catch (const std::exception& e) {
    return fail(e.what());
  }
  return SHZ_OK;
}

int shz_tree_neighbor(const shz_tree* t, int32_t level, const int32_t c[3], int32_t f, int32_t* kind, int32_t* v) {
  if (!t || !c || !kind || !v) return fail("shz_tree_neighbor: null argument");
  const int cc[3] = {c[0], c[1], c[2]};
  Block* b = t->t->get(level, cc);
  if (!b || f < 0 || f >= t->t->nface) return fail("shz_tree_neighbor: no such block or face");
  try {
    const auto nb = t->t->neighbor(b, f);
    *kind = nb.kind == shz::amr::NbKind::Same ? 0 : (nb.kind == shz::amr::NbKind::Coarse ? 1 : 2);
    *v = nb.kind == shz::amr::NbKind::Bc ? nb.type : nb.block->slot;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
  return SHZ_OK;
}

int shz_tree_table(const shz_tree* t, int32_t* out) {
  if (!t || !out) return fail("shz_tree_table: null argument");
  try {
    t->t->table(out);
  } catch (const std::exception& e) {
    return fail(e.what());
  }
  return SHZ_OK;
}

int shz_tree_lists(const shz_tree* t, int32_t* all, int32_t* leaves, int32_t* per_level, int32_t* n_all, int32_t* n_leaves) {
  if (!t) return fail("shz_tree_lists: null argument");
  std::vector<int32_t> a, l, p;
  t->t->lists(a, l, p);
  if (all) std::memcpy(all, a.data(), a.size() * sizeof(int32_t));
  if (leaves) std::memcpy(leaves, l.data(), l.size() * sizeof(int32_t));
  if (per_level) std::memcpy(per_level, p.data(), p.size() * sizeof(int32_t));
  if (n_all) *n_all = (int32_t)a.size();
  if (n_leaves) *n_leaves = (int32_t)l.size();
  return SHZ_OK;
}

int64_t shz_tree_index_grid_size(const shz_tree* t) { return t ? t->t->index_grid_size() : 0; }

int shz_tree_index_grid(const shz_tree* t, uint32_t* out) {
  if (!t || !out) return fail("shz_tree_index_grid: null argument");
  t->t->index_grid(out);
  return SHZ_OK;
}

int shz_tree_index_grid_boxes(shz_tree* t, uint32_t* out, int32_t* boxes, int32_t max_boxes, int32_t* n_boxes) {
  if (!t || !out || !n_boxes || (max_boxes > 0 && !boxes)) return fail("shz_tree_index_grid_boxes: null argument");
  std::vector<std::array<int, 6>> bx;
  const std::vector<uint32_t>& g = t->t->index_grid_tracked(&bx);
  std::memcpy(out, g.data(), g.size() * sizeof(uint32_t));
  *n_boxes = (int32_t)bx.size();
  for (int32_t i = 0; i < (int32_t)bx.size() && i < max_boxes; i++)
    for (int q = 0; q < 6; q++) boxes[6 * i + q] = bx[i][q];
  return SHZ_OK;
}

int shz_tree_set_bc(shz_tree* t, const int32_t bc_lo[3], const int32_t bc_hi[3]) {
  if (!t || !bc_lo || !bc_hi) return fail("shz_tree_set_bc: null argument");
  int lo[3], hi[3];
  for (int a = 0; a < 3; a++) { lo[a] = bc_lo[a]; hi[a] = bc_hi[a]; }
  t->t->set_bc(lo, hi);
  return SHZ_OK;
}

int shz_tree_stats(const shz_tree* t, int32_t* blocks, int32_t* free_slots, int32_t* leaves, int32_t* deepest, int32_t* high) {
  if (!t) return fail("shz_tree_stats: null argument");
  const auto lv = t->t->leaves();
  int d = 0;
  for (const Block* b : lv) d = std::max(d, b->level);
  if (blocks) *blocks = t->t->count();
  if (free_slots) *free_slots = t->t->free_slots();
  if (leaves) *leaves = (int32_t)lv.size();
  if (deepest) *deepest = d;
  if (high) *high = t->t->high_slot;
  return SHZ_OK;
}

}  // extern "C"
