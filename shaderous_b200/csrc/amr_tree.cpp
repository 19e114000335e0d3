// Host block tree: the decisions of the reference's src/amr/tree.ts, slot for slot.
// Citations are to that file. The reference keeps its tables up to date incrementally between
// re-meshes; the tables here are rebuilt whole on each read, which gives the same arrays (the
// reference's own test "keeps its block table and index grid up to date across re-meshes"
// asserts that equality).
#include "amr_tree.h"

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>

namespace shz {
namespace amr {

// tree.ts:139-184 constructor: the free stack holds cap-1 .. 0 with slot 0 on top, so slots are
// taken lowest first and a freed slot goes back on top.
BlockTree::BlockTree(int ndim_, int nr_, int max_level_, int cap_, const int lo[3], const int hi[3], bool edge,
                     const int* lim_)
    : ndim(ndim_), nr(nr_), max_level(max_level_), cap(cap_), level_limit(max_level_), nchild(1 << ndim_),
      nface(2 * ndim_), edge_balance(edge) {
  for (int a = 0; a < 3; a++) {
    bc_lo[a] = lo[a];
    bc_hi[a] = hi[a];
    lim[a] = lim_ ? lim_[a] : nr;
  }
  if (edge) {
    for (int a = 0; a < ndim; a++)
      for (int b = a + 1; b < ndim; b++)
        for (int sa : {-1, 1})
          for (int sb : {-1, 1}) {
            std::array<int, 3> d = {0, 0, 0};
            d[a] = sa;
            d[b] = sb;
            diagonals_.push_back(d);
          }
  }
  span_ = (int64_t)nr << max_level;
  slots_.assign(cap, nullptr);
  for (int s = cap - 1; s >= 0; s--) free_.push_back(s);
  const int nz = ndim == 3 ? lim[2] : 1;
  const int nroot = lim[0] * (ndim >= 2 ? lim[1] : 1) * nz;
  if (nroot > cap)
    throw std::runtime_error("block budget " + std::to_string(cap) + " is smaller than the " + std::to_string(nroot) +
                             " root blocks");
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < (ndim >= 2 ? lim[1] : 1); j++)
      for (int i = 0; i < lim[0]; i++) {
        const int c[3] = {i, j, k};
        create(0, c, nullptr);
      }
}

int64_t BlockTree::key(int level, int c0, int c1, int c2) const {
  return (((int64_t)level * span_ + c2) * span_ + c1) * span_ + c0;
}

Block* BlockTree::create(int level, const int c[3], Block* parent) {
  const int slot = free_.back();
  free_.pop_back();
  if (slot > high_slot) high_slot = slot;
  arena_.push_back(Block{slot, level, {c[0], c[1], c[2]}, parent, {}});
  Block* b = &arena_.back();
  ++version_;
  slots_[slot] = b;
  blocks_[key(level, c[0], c[1], c[2])] = b;
  new_leaves_.push_back(b);  // tree.ts:234
  return b;
}

void BlockTree::remove(Block* b) {
  blocks_.erase(key(b->level, b->c[0], b->c[1], b->c[2]));
  ++version_;
  slots_[b->slot] = nullptr;
  free_.push_back(b->slot);
}

bool BlockTree::live(const Block* b) const {
  auto it = blocks_.find(key(b->level, b->c[0], b->c[1], b->c[2]));
  return it != blocks_.end() && it->second == b;
}

std::vector<Block*> BlockTree::all() const {
  std::vector<std::vector<Block*>> by(max_level + 1);
  for (Block* b : slots_)
    if (b) by[b->level].push_back(b);
  std::vector<Block*> out;
  for (auto& v : by) out.insert(out.end(), v.begin(), v.end());
  return out;
}

std::vector<Block*> BlockTree::leaves() const {
  std::vector<Block*> out;
  for (Block* b : all())
    if (b->leaf()) out.push_back(b);
  return out;
}

Block* BlockTree::get(int level, const int c[3]) const {
  auto it = blocks_.find(key(level, c[0], c[1], ndim == 3 ? c[2] : 0));
  return it == blocks_.end() ? nullptr : it->second;
}

// tree.ts:283-304 neighbor.
Neighbor BlockTree::neighbor(const Block* b, int f) const {
  const int axis = f >> 1;
  int c[3] = {b->c[0], b->c[1], b->c[2]};
  const int step = (f & 1) ? 1 : -1;
  const int n = lim[axis] << b->level;
  int v = c[axis] + step;
  if (v < 0 || v >= n) {
    const int type = (f & 1) ? bc_hi[axis] : bc_lo[axis];
    if (type != 0) return {NbKind::Bc, nullptr, type};
    v = (v + n) % n;
  }
  c[axis] = v;
  auto it = blocks_.find(key(b->level, c[0], c[1], c[2]));
  if (it != blocks_.end()) return {NbKind::Same, it->second, 0};
  if (b->level > 0) {
    auto co = blocks_.find(key(b->level - 1, c[0] >> 1, c[1] >> 1, c[2] >> 1));
    if (co != blocks_.end()) return {NbKind::Coarse, co->second, 0};
  }
  throw std::runtime_error("2:1 balance broken at level " + std::to_string(b->level) + " face " + std::to_string(f));
}

// tree.ts:311-329 atOffset.
Block* BlockTree::at_offset(const Block* b, const int d[3]) const {
  int c[3] = {b->c[0], b->c[1], b->c[2]};
  for (int a = 0; a < 3; a++) {
    if (!d[a]) continue;
    const int n = lim[a] << b->level;
    int v = c[a] + d[a];
    if (v < 0 || v >= n) {
      if ((d[a] > 0 ? bc_hi[a] : bc_lo[a]) != 0) return nullptr;
      v = (v + n) % n;
    }
    c[a] = v;
  }
  for (int l = b->level; l >= 0; l--) {
    const int s = b->level - l;
    auto it = blocks_.find(key(l, c[0] >> s, c[1] >> s, c[2] >> s));
    if (it != blocks_.end()) return it->second;
  }
  return nullptr;
}

// tree.ts:332-343 coarserAround.
std::vector<Block*> BlockTree::coarser_around(const Block* b) const {
  std::vector<Block*> out;
  for (int f = 0; f < nface; f++) {
    Neighbor nb = neighbor(b, f);
    if (nb.kind == NbKind::Coarse) out.push_back(nb.block);
  }
  for (const auto& d : diagonals_) {
    Block* q = at_offset(b, d.data());
    if (q && q->level < b->level) out.push_back(q);
  }
  return out;
}

// tree.ts:346-352 refineCost.
template <class Set>
int BlockTree::refine_cost(const Block* b, Set& seen) const {
  if (seen.count(b) || !b->leaf()) return 0;
  seen.insert(b);
  int cost = nchild;
  for (Block* q : coarser_around(b)) cost += refine_cost(q, seen);
  return cost;
}

int BlockTree::cost_to_refine(const std::vector<Block*>& list) const {
  std::unordered_set<const Block*> seen;
  int cost = 0;
  for (Block* b : list) cost += refine_cost(b, seen);
  return cost;
}

// tree.ts:366-386 refine: split a leaf, first splitting coarser neighbours so balance holds.
std::vector<Block*> BlockTree::refine(Block* b, const std::unordered_set<Block*>* forbidden,
                                      BlockSet* need_out, int* cost_out) {
  std::vector<Block*> done;
  if (!b->leaf() || b->level >= level_limit) return done;
  BlockSet need;
  const int cost = refine_cost(b, need);
  if (cost > (int)free_.size()) {
    if (need_out) *need_out = std::move(need);
    if (cost_out) *cost_out = cost;
    return done;
  }
  if (forbidden)
    for (const Block* q : need)
      if (forbidden->count(const_cast<Block*>(q))) return done;
  std::function<void(Block*)> split = [&](Block* q) {
    if (!q->leaf()) return;
    const std::vector<Block*> around = coarser_around(q);
    for (Block* nb : around) split(nb);
    if (!q->leaf()) return;
    q->children.reserve(nchild);
    for (int o = 0; o < nchild; o++) {
      const int c[3] = {2 * q->c[0] + (o & 1), 2 * q->c[1] + ((o >> 1) & 1), ndim == 3 ? 2 * q->c[2] + ((o >> 2) & 1) : 0};
      q->children.push_back(create(q->level + 1, c, q));
    }
    done.push_back(q);
  };
  split(b);
  return done;
}

// tree.ts:389-402 canCoarsen.
bool BlockTree::can_coarsen(const Block* p) const {
  if (p->leaf()) return false;
  for (const Block* ch : p->children)
    if (!ch->leaf()) return false;
  for (const Block* ch : p->children) {
    for (int f = 0; f < nface; f++) {
      Neighbor nb = neighbor(ch, f);
      if (nb.kind == NbKind::Same && !nb.block->leaf()) return false;
    }
    for (const auto& d : diagonals_) {
      const Block* q = at_offset(ch, d.data());
      if (q && q->level == ch->level && !q->leaf()) return false;
    }
  }
  return true;
}

// tree.ts:404-409 coarsen.
void BlockTree::coarsen(Block* p) {
  for (Block* ch : p->children) remove(ch);
  p->children.clear();
  new_leaves_.push_back(p);  // tree.ts:417
}

// tree.ts:420-430 evictable: parents with only leaf children, scored by their most strongly
// flagged child; the lowest tier first, then the least flagged (a stable sort, as Array.sort).
std::vector<BlockTree::Evictable> BlockTree::evictable(const std::vector<Block*>& lv, const SlotVals& ind,
                                                       const std::function<double(const Block*)>& tier) const {
  std::vector<Block*> parents;
  std::unordered_set<const Block*> seen;
  for (Block* b : lv)
    if (b->parent && seen.insert(b->parent).second) parents.push_back(b->parent);
  std::vector<Evictable> out;
  for (Block* p : parents) {
    if (p->leaf()) continue;
    bool any = false;
    for (Block* ch : p->children) any |= !ch->leaf();
    if (any) continue;
    double score = -std::numeric_limits<double>::infinity();
    for (Block* ch : p->children) score = std::max(score, ind.get(ch, 0.0));
    out.push_back({p, score, tier ? tier(p) : NO_TIER});
  }
  std::stable_sort(out.begin(), out.end(), [](const Evictable& a, const Evictable& b) {
    if (a.tier == b.tier) return a.score < b.score;
    return a.tier > b.tier;
  });
  return out;
}

// tree.ts:433-442 near.
bool BlockTree::near(const Block* a, const Block* q) const {
  const int64_t sa = (int64_t)1 << (max_level - a->level);
  const int64_t sq = (int64_t)1 << (max_level - q->level);
  for (int i = 0; i < ndim; i++) {
    const int64_t lo = a->c[i] * sa;
    const int64_t qlo = (q->c[i] - 1) * sq;
    if (lo + sa <= qlo || qlo + 3 * sq <= lo) return false;
  }
  return true;
}

// tree.ts:449-467 makeRoom. The candidates' tests are the reference's, in its order; those that
// do not involve b (touched, live, leaf children, canCoarsen) are pure functions of the tree and
// the touched set, which change together, so they are evaluated once per version of the tree and
// the candidates that failed them are not visited again: adapt calls this for every flagged leaf,
// and on a full slot budget each call would scan thousands of candidates. The stopping test (tier
// and score against b's) holds from some candidate on, in the sorted order, so checking it at the
// candidates that pass stops where the full scan would (the ones in between add nothing).
bool BlockTree::make_room(Block* b, double level, const std::vector<Evictable>& ev,
                          const std::unordered_set<const Block*>& touched, double tier, std::vector<Block*>& out,
                          EvictCache& cache, const BlockSet* need_in, int cost_in) {
  out.clear();
  if (!b->leaf() || b->level >= level_limit) return false;
  BlockSet own;
  const BlockSet& need = need_in ? *need_in : own;
  int shortage = (need_in ? cost_in : refine_cost(b, own)) - (int)free_.size();
  if (shortage <= 0) return false;
  if (cache.version != version_) {
    cache.ok_idx.clear();
    cache.evaluated = 0;
    cache.version = version_;
  }
  auto stop = [&](const Evictable& e) { return e.tier < tier || (e.tier == tier && e.score >= EVICT_MARGIN * level); };
  size_t k = 0;
  for (;;) {
    size_t i;
    if (k < cache.ok_idx.size()) {
      i = (size_t)cache.ok_idx[k++];
      if (stop(ev[i])) break;
    } else {
      if (cache.evaluated >= ev.size()) break;
      i = cache.evaluated;
      if (stop(ev[i])) break;
      cache.evaluated++;
      Block* p = ev[i].p;
      bool ok = !(touched.count(p) || !live(p) || p->leaf());
      if (ok)
        for (Block* ch : p->children) ok = ok && ch->leaf() && touched.count(ch) == 0;
      ok = ok && can_coarsen(p);
      if (!ok) continue;
      cache.ok_idx.push_back((int)i);
      k = cache.ok_idx.size();
    }
    Block* p = ev[i].p;
    if (need.count(p)) continue;
    bool close = false;
    for (const Block* q : need)
      if (near(p, q)) { close = true; break; }
    if (close) continue;
    out.push_back(p);
    shortage -= nchild;
    if (shortage <= 0) return true;
  }
  out.clear();
  return false;
}

namespace {
// tree.ts:598-636 adaptRun: the bookkeeping of a re-mesh.
struct Run {
  BlockTree& t;
  std::unordered_set<const Block*>& touched;
  std::unordered_map<int, RegridOp> ops;
  std::vector<std::vector<int>> steps;
  std::unordered_set<Block*> evicted;

  void merge(Block* p) {
    RegridOp op;
    op.kind = RG_RESTRICT;
    op.src = p->slot;
    for (Block* ch : p->children) op.children.push_back(ch->slot);
    if (t.ndim == 1) {
      const std::vector<int> c = op.children;
      op.children.insert(op.children.end(), c.begin(), c.end());
    }
    t.coarsen(p);
    touched.insert(p);
    ops[p->slot] = op;
  }
  // (refine: the blocks a failed split would take, for make_room)
  BlockSet need;
  int cost = -1;
  bool step(int what, Block* b) {
    std::vector<int> s = {what, b->level};
    for (int a = 0; a < t.ndim; a++) s.push_back(b->c[a]);
    steps.push_back(s);
    if (what == ADAPT_REFINE) {
      cost = -1;
      const std::vector<Block*> split = t.refine(b, &evicted, &need, &cost);
      for (Block* q : split) {
        touched.insert(q);
        for (int o = 0; o < (int)q->children.size(); o++) {
          touched.insert(q->children[o]);
          RegridOp op;
          op.kind = RG_PROLONG;
          op.src = q->slot;
          op.octant = o;
          ops[q->children[o]->slot] = op;
        }
      }
      return !split.empty();
    }
    merge(b);
    if (what == ADAPT_EVICT) evicted.insert(b);
    return true;
  }
  std::vector<RegridOp> table() {
    std::vector<RegridOp> out;
    if (ops.empty()) return out;
    out.assign(t.cap, RegridOp());
    for (Block* leaf : t.leaves()) {
      auto it = ops.find(leaf->slot);
      if (it != ops.end()) {
        out[leaf->slot] = it->second;
      } else {
        RegridOp op;
        op.kind = RG_COPY;
        op.src = leaf->slot;
        out[leaf->slot] = op;
      }
    }
    return out;
  }
};
}  // namespace

// tree.ts:489-544 adapt.
std::vector<RegridOp> BlockTree::adapt(const std::function<double(const Block*)>& indicator, double hi, double lo,
                                       const std::function<double(const Block*)>& tier) {
  const std::vector<Block*> before = leaves();
  SlotVals ind, tiers;
  ind.init(cap);
  tiers.init(cap);
  for (Block* b : before) {
    const double t = tier ? tier(b) : NO_TIER;
    tiers.set(b, t);
    const double raw = indicator(b);
    ind.set(b, (t < NO_TIER && raw >= 0) ? std::max(raw, ZONE_INDICATOR) : raw);
  }
  std::unordered_set<const Block*> touched;
  Run run{*this, touched, {}, {}, {}};

  std::vector<Block*> wanted;
  for (Block* b : before)
    if (ind.get(b, 0.0) > hi && b->level < level_limit) wanted.push_back(b);
  std::stable_sort(wanted.begin(), wanted.end(), [&](Block* a, Block* b) {
    const double ta = tiers.get(a, NO_TIER), tb = tiers.get(b, NO_TIER);
    if (ta == tb) return ind.get(a, 0.0) > ind.get(b, 0.0);
    return ta < tb;
  });
  bool have_ev = false;
  std::vector<Evictable> ev;
  EvictCache ev_cache;
  std::vector<Block*> room;
  for (Block* b : wanted) {
    if (!b->leaf() || !live(b)) continue;
    if (!run.step(ADAPT_REFINE, b)) {
      if (!have_ev) {
        ev = evictable(before, ind, tier);
        have_ev = true;
      }
      // (the failed split's own count, if it got that far: make_room needs the same at this version)
      const bool known = run.cost >= 0;
      if (make_room(b, ind.get(b, 0.0), ev, touched, tiers.get(b, NO_TIER), room, ev_cache, known ? &run.need : nullptr,
                    run.cost)) {
        for (Block* p : room) run.step(ADAPT_EVICT, p);
        run.step(ADAPT_REFINE, b);
      }
    }
  }

  auto ind_of = [&](const Block* b) { return ind.get(b, 0.0); };
  auto hot = [&](const Block* b) {
    if (ind_of(b) > lo) return true;
    if (tiers.has(b) && tiers.get(b, NO_TIER) < NO_TIER) return true;
    if (ind_of(b) < 0) return false;
    for (int f = 0; f < nface; f++) {
      Neighbor nb = neighbor(b, f);
      if (nb.kind != NbKind::Bc && ind_of(nb.block) > hi) return true;
    }
    return false;
  };
  std::vector<Block*> parents;
  std::unordered_set<const Block*> seen;
  for (Block* b : before)
    if (b->parent && seen.insert(b->parent).second) parents.push_back(b->parent);
  for (Block* p : parents) {
    if (touched.count(p) || !live(p) || p->leaf()) continue;
    bool skip = false;
    for (Block* ch : p->children) skip |= touched.count(ch) > 0 || !ch->leaf();
    if (skip) continue;
    bool any_hot = false;
    for (Block* ch : p->children)
      if (hot(ch)) { any_hot = true; break; }
    if (any_hot || !can_coarsen(p)) continue;
    run.step(ADAPT_MERGE, p);
  }
  last_steps = run.steps;
  return run.table();
}

// tree.ts:579-589 replayAdapt.
std::vector<RegridOp> BlockTree::replay_adapt(const std::vector<std::vector<int>>& steps) {
  std::unordered_set<const Block*> touched;
  Run run{*this, touched, {}, {}, {}};
  for (const auto& s : steps) {
    int c[3] = {0, 0, 0};
    for (int a = 0; a < ndim; a++) c[a] = s[2 + a];
    Block* b = get(s[1], c);
    if (!b) throw std::runtime_error("a re-mesh to replay acts on a block the mesh does not have");
    run.step(s[0], b);
  }
  last_steps = run.steps;
  return run.table();
}

// tree.ts:654-679 writeRow, for every slot.
void BlockTree::table(int32_t* t) const {
  for (int slot = 0; slot < cap; slot++) {
    int32_t* o = t + (size_t)slot * BT_STRIDE;
    for (int i = 0; i < BT_STRIDE; i++) o[i] = -1;
    o[4] = 0;
    const Block* b = slots_[slot];
    if (!b) continue;
    o[0] = b->level;
    o[1] = b->c[0];
    o[2] = b->c[1];
    o[3] = b->c[2];
    o[4] = FLAG_ACTIVE | (b->leaf() ? FLAG_LEAF : 0);
    o[5] = b->parent ? b->parent->slot : -1;
    for (int f = 0; f < 6; f++) {
      if (f >= nface) {
        o[6 + f] = b->slot;
        continue;
      }
      Neighbor nb = neighbor(b, f);
      if (nb.kind == NbKind::Same) {
        o[6 + f] = nb.block->slot;
      } else if (nb.kind == NbKind::Coarse) {
        o[6 + f] = NB_COARSE;
        o[20 + f] = nb.block->slot;
      } else {
        o[6 + f] = -1 - nb.type;
      }
    }
    for (size_t i = 0; i < b->children.size(); i++) o[12 + i] = b->children[i]->slot;
    if (!b->leaf() && ndim == 1)
      for (size_t i = 0; i < b->children.size(); i++) o[14 + i] = b->children[i]->slot;
  }
}

// tree.ts:681-693 regridTable.
void BlockTree::regrid_table(const std::vector<RegridOp>& ops, int cap, int32_t* t) {
  std::memset(t, 0, sizeof(int32_t) * (size_t)cap * RG_STRIDE);
  for (int slot = 0; slot < (int)ops.size() && slot < cap; slot++) {
    const RegridOp& op = ops[slot];
    if (op.kind == RG_NONE) continue;
    int32_t* o = t + (size_t)slot * RG_STRIDE;
    o[0] = op.kind;
    o[1] = op.src;
    o[2] = op.octant;
    for (size_t i = 0; i < op.children.size() && i < 8; i++) o[4 + i] = op.children[i];
  }
}

// tree.ts:695-715 lists.
void BlockTree::lists(std::vector<int32_t>& a, std::vector<int32_t>& lv, std::vector<int32_t>& per_level) const {
  a.clear();
  lv.clear();
  per_level.assign(max_level + 1, 0);
  for (const Block* b : all()) {
    a.push_back(b->slot);
    per_level[b->level]++;
    if (b->leaf()) lv.push_back(b->slot);
  }
}

int64_t BlockTree::index_grid_size() const {
  const int64_t m = (int64_t)nr << max_level;
  return ndim == 1 ? m : (ndim == 2 ? m * m : m * m * m);
}

// tree.ts:805-812 fillLeaf: a leaf's cells of the index grid.
void BlockTree::fill_leaf(uint32_t* g, const Block* b) const {
  const int64_t m = (int64_t)nr << max_level;
  const int64_t span = (int64_t)1 << (max_level - b->level);
  if (ndim == 1) {
    for (int64_t x = b->c[0] * span; x < (b->c[0] + 1) * span; x++) g[x] = b->slot;
    return;
  }
  const int64_t z0 = ndim == 3 ? b->c[2] * span : 0;
  for (int64_t k = z0; k < z0 + (ndim == 3 ? span : 1); k++)
    for (int64_t j = b->c[1] * span; j < (b->c[1] + 1) * span; j++)
      for (int64_t x = b->c[0] * span; x < (b->c[0] + 1) * span; x++) g[(k * m + j) * m + x] = b->slot;
}

// tree.ts:721-816 indexGrid (the whole grid; every cell lies in exactly one leaf).
void BlockTree::index_grid(uint32_t* g) const {
  for (const Block* b : slots_)
    if (b && b->leaf()) fill_leaf(g, b);
}

// tree.ts:721-803 indexGrid with boxes: filling the leaves made since the last read covers
// whatever changed (every cell lies in exactly one leaf). The boxes: per row of the outer axis (y
// in 2D, z in 3D) the extent filled along the inner ones, merged into runs of rows that bridge
// gaps of up to GAP = 4 unchanged rows (each box costs the caller a copy call).
const std::vector<uint32_t>& BlockTree::index_grid_tracked(std::vector<std::array<int, 6>>* boxes) {
  const int m = nr << max_level;
  const bool d3 = ndim == 3;
  const int mz = d3 ? m : 1;
  const size_t n = (size_t)index_grid_size();
  if (grid_.size() != n) {
    grid_.assign(n, 0u);
    index_grid(grid_.data());
    new_leaves_.clear();
    if (boxes) boxes->push_back({0, 0, 0, m, ndim >= 2 ? m : 1, mz});
    return grid_;
  }
  if (ndim == 1) {
    int lo = m, hi = 0;
    for (Block* b : new_leaves_) {
      if (!b->leaf() || slots_[b->slot] != b) continue;
      fill_leaf(grid_.data(), b);
      const int span = 1 << (max_level - b->level);
      lo = std::min(lo, b->c[0] * span);
      hi = std::max(hi, (b->c[0] + 1) * span);
    }
    new_leaves_.clear();
    if (boxes && hi > lo) boxes->push_back({lo, 0, 0, hi - lo, 1, 1});
    return grid_;
  }
  std::vector<int> lo0(m, m), hi0(m, 0), lo1(m, m), hi1(m, 0);
  for (Block* b : new_leaves_) {
    if (!b->leaf() || slots_[b->slot] != b) continue;
    fill_leaf(grid_.data(), b);
    const int span = 1 << (max_level - b->level);
    const int x0 = b->c[0] * span, y0 = b->c[1] * span, o0 = (d3 ? b->c[2] : b->c[1]) * span;
    for (int o = o0; o < o0 + span; o++) {
      lo0[o] = std::min(lo0[o], x0);
      hi0[o] = std::max(hi0[o], x0 + span);
      if (d3) {
        lo1[o] = std::min(lo1[o], y0);
        hi1[o] = std::max(hi1[o], y0 + span);
      }
    }
  }
  new_leaves_.clear();
  if (!boxes) return grid_;
  constexpr int GAP = 4;
  for (int o = 0; o < m;) {
    if (hi0[o] == 0) {
      o++;
      continue;
    }
    int a0 = m, b0 = 0, a1 = m, b1 = 0, end = o;
    for (int k = o; k < m && k <= end + GAP; k++) {
      if (hi0[k] == 0) continue;
      a0 = std::min(a0, lo0[k]);
      b0 = std::max(b0, hi0[k]);
      a1 = std::min(a1, lo1[k]);
      b1 = std::max(b1, hi1[k]);
      end = k;
    }
    if (d3) boxes->push_back({a0, a1, o, b0 - a0, b1 - a1, end + 1 - o});
    else boxes->push_back({a0, o, 0, b0 - a0, end + 1 - o, 1});
    o = end + 1;
  }
  return grid_;
}

void BlockTree::set_bc(const int lo[3], const int hi[3]) {
  for (int a = 0; a < 3; a++) {
    bc_lo[a] = lo[a];
    bc_hi[a] = hi[a];
  }
  ++version_;  // cached neighbour tests see a new tree
}

}  // namespace amr
}  // namespace shz
