// The block tree of the adaptive grid, on the host: a restatement of the reference's
// src/amr/tree.ts (BlockTree) that makes the same decisions slot for slot given the same
// indicators, and writes the same flat tables the GPU passes read.
//
// The domain is covered by lim[0] x lim[1] (x lim[2]) root blocks of BS^ndim cells. A block
// splits into 2^ndim children of half the cell size; leaves carry the solution and parents
// nothing. Face neighbours never differ by more than one level (2:1 balance), and with
// edge_balance the same holds across edges (3D) or vertices (2D).
#pragma once
#include <array>
#include <cstdint>
#include <deque>
#include <functional>
#include <limits>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace shz {
namespace amr {

constexpr int BS = 16;          // cells per block side (tree.ts:14)
constexpr int MAX_LEVELS = 7;   // tree.ts:16
constexpr int NG = 2;           // ghost layers (tree.ts:17)
constexpr int PAD = BS + 2 * NG;
constexpr int BT_STRIDE = 32;   // ints per block in the block table (tree.ts:19)
constexpr int RG_STRIDE = 12;   // ints per block in the regrid table (tree.ts:20)
constexpr int NB_COARSE = -1;   // tree.ts:52
constexpr int FLAG_ACTIVE = 1, FLAG_LEAF = 2;
constexpr int RG_NONE = 0, RG_COPY = 1, RG_PROLONG = 2, RG_RESTRICT = 3;  // tree.ts:63-66
constexpr int ADAPT_REFINE = 0, ADAPT_EVICT = 1, ADAPT_MERGE = 2;        // tree.ts:95-99
constexpr double EVICT_MARGIN = 0.8;                                      // tree.ts:106
constexpr double ZONE_INDICATOR = 1e30;                                   // tree.ts:113
constexpr double NO_TIER = std::numeric_limits<double>::infinity();

struct Block {
  int slot;
  int level;
  int c[3];
  Block* parent;
  std::vector<Block*> children;  // empty: a leaf
  bool leaf() const { return children.empty(); }
};

// A set of the few blocks one refinement takes (a leaf and the coarser neighbours balance splits
// with it), searched linearly: cheaper than a hash set at that size, and adapt asks for one per
// flagged leaf.
struct BlockSet {
  std::vector<const Block*> v;
  size_t count(const Block* b) const {
    for (const Block* x : v)
      if (x == b) return 1;
    return 0;
  }
  bool insert(const Block* b) {
    if (count(b)) return false;
    v.push_back(b);
    return true;
  }
  std::vector<const Block*>::const_iterator begin() const { return v.begin(); }
  std::vector<const Block*>::const_iterator end() const { return v.end(); }
};

struct RegridOp {
  int kind = RG_NONE;
  int src = -1;
  int octant = 0;
  std::vector<int> children;
};

enum class NbKind { Same, Coarse, Bc };
struct Neighbor {
  NbKind kind;
  Block* block;  // Same / Coarse
  int type;      // Bc
};

class BlockTree {
 public:
  BlockTree(int ndim, int nr, int max_level, int cap, const int bc_lo[3], const int bc_hi[3], bool edge_balance = false,
            const int* lim = nullptr);

  const int ndim, nr, max_level, cap;
  int level_limit;
  const int nchild, nface;
  const bool edge_balance;
  int lim[3];
  int bc_lo[3], bc_hi[3];
  int high_slot = -1;

  int count() const { return cap - (int)free_.size(); }
  int free_slots() const { return (int)free_.size(); }
  const std::vector<Block*>& slots() const { return slots_; }

  std::vector<Block*> all() const;     // coarsest first, by slot within a level
  std::vector<Block*> leaves() const;
  Block* get(int level, const int c[3]) const;
  Neighbor neighbor(const Block* b, int f) const;
  Block* at_offset(const Block* b, const int d[3]) const;
  // need_out / cost_out (if given): the blocks the split would take and their slots, once computed
  // (a refinement that fails for want of slots hands them on to make_room).
  std::vector<Block*> refine(Block* b, const std::unordered_set<Block*>* forbidden = nullptr,
                             BlockSet* need_out = nullptr, int* cost_out = nullptr);
  bool can_coarsen(const Block* p) const;
  void coarsen(Block* p);
  int cost_to_refine(const std::vector<Block*>& list) const;

  // Re-mesh from an indicator per leaf (tree.ts:489-544); tier: refinement zones (NO_TIER for
  // none). Returns the regrid ops per slot of the new tree (cap entries), or an empty vector if
  // nothing changed.
  std::vector<RegridOp> adapt(const std::function<double(const Block*)>& indicator, double hi, double lo,
                              const std::function<double(const Block*)>& tier = nullptr);
  std::vector<RegridOp> replay_adapt(const std::vector<std::vector<int>>& steps);
  std::vector<std::vector<int>> last_steps;

  void table(int32_t* out) const;  // cap * BT_STRIDE ints (tree.ts:642-679)
  static void regrid_table(const std::vector<RegridOp>& ops, int cap, int32_t* out);  // cap * RG_STRIDE
  // Slot lists: every block (coarsest first) and the leaves; counts per level.
  void lists(std::vector<int32_t>& all, std::vector<int32_t>& leaves, std::vector<int32_t>& per_level) const;
  void index_grid(uint32_t* out) const;  // (nr << max_level)^ndim leaf slots (tree.ts:721)
  int64_t index_grid_size() const;
  // tree.ts:721-803 indexGrid(boxes): the index grid kept between reads, updated from the leaves
  // made since the last read, and the boxes (origin, size; 6 ints each) that cover what changed:
  // the whole grid on the first read, else runs of changed rows of the outer axis.
  const std::vector<uint32_t>& index_grid_tracked(std::vector<std::array<int, 6>>* boxes);
  // tree.ts:193-199 the bcLo / bcHi setters: boundary types of a tree already built (every table
  // read after the change shows them).
  void set_bc(const int lo[3], const int hi[3]);

 private:
  std::vector<uint32_t> grid_;       // the index grid as last read (empty: not read yet)
  std::vector<Block*> new_leaves_;   // blocks that became leaves since the last read (tree.ts:129)
  void fill_leaf(uint32_t* g, const Block* b) const;
  int64_t key(int level, int c0, int c1, int c2) const;
  Block* create(int level, const int c[3], Block* parent);
  void remove(Block* b);
  bool live(const Block* b) const;
  Block* same_level(const Block* b, int f) const;
  std::vector<Block*> coarser_around(const Block* b) const;
  template <class Set>
  int refine_cost(const Block* b, Set& seen) const;
  struct Evictable {
    Block* p;
    double score;
    double tier;
  };
  // A value per block, held by slot with the block it belongs to (a slot freed and taken again in
  // one re-mesh belongs to another block: blocks are never reused, so identity tells them apart).
  struct SlotVals {
    std::vector<const Block*> who;
    std::vector<double> v;
    void init(int n) {
      who.assign(n, nullptr);
      v.assign(n, 0.0);
    }
    void set(const Block* b, double x) {
      who[b->slot] = b;
      v[b->slot] = x;
    }
    bool has(const Block* b) const { return who[b->slot] == b; }
    double get(const Block* b, double dflt) const { return who[b->slot] == b ? v[b->slot] : dflt; }
  };
  std::vector<Evictable> evictable(const std::vector<Block*>& leaves, const SlotVals& ind,
                                   const std::function<double(const Block*)>& tier) const;
  bool near(const Block* a, const Block* q) const;
  // The part of make_room's test of a candidate that does not depend on the block being refined,
  // for one version of the tree (recomputed when the tree has changed): the entries of `ev` below
  // `evaluated` have been tested, and ok_idx lists those that passed, in order.
  struct EvictCache {
    std::vector<int> ok_idx;
    size_t evaluated = 0;
    uint64_t version = ~0ull;
  };
  // need / cost: b's refine_cost set and count if already computed at this version (else null).
  bool make_room(Block* b, double level, const std::vector<Evictable>& ev, const std::unordered_set<const Block*>& touched,
                 double tier, std::vector<Block*>& out, EvictCache& cache,
                 const BlockSet* need = nullptr, int cost = 0);

  std::deque<Block> arena_;  // blocks are never freed while the tree lives (identity for live())
  std::unordered_map<int64_t, Block*> blocks_;
  std::vector<Block*> slots_;
  std::vector<int> free_;  // a stack: back() is the top
  uint64_t version_ = 0;   // bumped by every create and remove
  int64_t span_;
  std::vector<std::array<int, 3>> diagonals_;
};

}  // namespace amr
}  // namespace shz
