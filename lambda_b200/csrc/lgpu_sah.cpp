// lgpu_sah.cpp — the traversal tree of a mesh: an 8-wide BVH built with the
// surface-area heuristic, in the reference's own node format (cg.hpp:596-631)
// so that it is laid out for the device like the reference's tree.
//
// The reference's builder (bvh::build, cg.hpp:632-749) splits every node
// into 8 equal-width centroid bins along its longest axis, so a node's
// children are slabs along one axis; a ray crosses many of them.  Here a
// binary tree is built top-down, each range split where the surface-area
// cost (the area-weighted primitive counts of the two sides) is lowest: over
// 32 centroid bins on the axis of the largest centroid extent (binning all
// three axes took 2.1x the build time for a tree that traced no faster; 32
// bins traced 0.45 % faster than 16, measured), or, for at most 24
// primitives, over every split of their centroid order on each axis.  The
// binary tree is then collapsed into wide nodes of up to 8 children and
// leaves of up to max_leaf primitives by the cost-optimal dynamic program
// of Ylitie, Karras and Laine (HPG 2017): frame +1.2 % against opening the
// child of largest area until there are 8, measured.  The closest hit along
// a ray does not depend on the tree (the triangle test is the same exact
// test); only which of two faces at exactly equal distance is reported can.
// The reference's own tree is kept for the reference-order traversal.
//
// A binned split visits its primitives twice: once to bin them, once to
// partition them (the children's centroid bounds on the way); the
// children's boxes come from the bins.  Subtrees of more than kSpawn
// primitives are queued for the worker threads, each of which keeps the
// nodes it builds and costs them on the way up.
#include <algorithm>
#include <atomic>
#include <exception>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "lgpu_layout.h"

namespace lgpu {

namespace {

constexpr int kBins = 32;

struct Box {
  float lo[3], hi[3];
  void init() {
    for (int k = 0; k < 3; k++) {
      lo[k] = 1e30f;
      hi[k] = -1e30f;
    }
  }
  void add(const Box& b) {
    for (int k = 0; k < 3; k++) {
      lo[k] = std::min(lo[k], b.lo[k]);
      hi[k] = std::max(hi[k], b.hi[k]);
    }
  }
  double area() const {
    double const dx = std::max(0.0, double(hi[0]) - lo[0]), dy = std::max(0.0, double(hi[1]) - lo[1]),
                 dz = std::max(0.0, double(hi[2]) - lo[2]);
    return dx * dy + dy * dz + dz * dx;
  }
};

// primitives prims[b, e), the union of their boxes and the bounds of their
// centroids
struct Range {
  uint32_t b, e;
  Box box, cbox;
  uint32_t size() const { return e - b; }
};

// A node of the binary build tree over primitives prims[b, e): one
// primitive, or two children referenced as (worker << 24) | index in that
// worker's nodes.  C[i] is the least cost of the subtree as at most i + 1
// roots of wide nodes or leaves (the dynamic program of Ylitie, Karras and
// Laine, "Efficient Incoherent Ray Traversal on GPUs Through Compressed
// Wide BVHs", HPG 2017), with the choice that reaches it: D[i] = kOneLeaf
// or kOneNode (one root: this node as a leaf, or as a wide node whose
// children split 8 roots K[0] / 8 - K[0] between its two children),
// kSplit (K[i] roots from the first child, the rest from the second) or
// kFewer (as with i roots).
enum : uint8_t { kOneLeaf = 0, kOneNode = 1, kSplit = 2, kFewer = 3 };
struct BNode {
  Box box;
  uint32_t b = 0, e = 0;
  uint32_t kid[2] = {0, 0};
  bool leaf = false;    // a single primitive
  bool costed = false;  // C, D and K are set
  float C[8];
  uint8_t D[8], K[8];
};
constexpr uint32_t kLocalBits = 24;
// the costs of the dynamic program: a wide node's box tests and a leaf's
// triangle tests per unit of surface area (the best of the costs measured:
// 0.3 against 0.5 per face, leaves of at most 2 faces against 3)
constexpr float kCostNode = 1.f, kCostFace = 0.3f, kCostInf = 1e30f;

// C, D and K of nd from its children's
void dp_cost(BNode& nd, const BNode* kid0, const BNode* kid1, size_t max_leaf) {
  uint32_t const n = nd.e - nd.b;
  float const area = float(nd.box.area());
  float const leaf = n <= max_leaf ? area * kCostFace * float(n) : kCostInf;
  if (nd.leaf) {
    for (int i = 0; i < 8; i++) {
      nd.C[i] = leaf;
      nd.D[i] = i == 0 ? kOneLeaf : kFewer;
      nd.K[i] = 0;
    }
    nd.costed = true;
    return;
  }
  // dist[j - 1]: the least cost of j roots split between the children
  float dist[8];
  uint8_t dk[8];
  for (int j = 0; j < 8; j++) {
    dist[j] = kCostInf;
    dk[j] = 0;
  }
  for (int j = 2; j <= 8; j++)
    for (int k = 1; k < j; k++) {
      float const v = kid0->C[k - 1] + kid1->C[j - k - 1];
      if (v < dist[j - 1]) {
        dist[j - 1] = v;
        dk[j - 1] = uint8_t(k);
      }
    }
  float const node = area * kCostNode + dist[7];
  if (leaf <= node) {
    nd.C[0] = leaf;
    nd.D[0] = kOneLeaf;
    nd.K[0] = 0;
  } else {
    nd.C[0] = node;
    nd.D[0] = kOneNode;
    nd.K[0] = dk[7];
  }
  for (int i = 2; i <= 8; i++) {
    if (dist[i - 1] < nd.C[i - 2]) {
      nd.C[i - 1] = dist[i - 1];
      nd.D[i - 1] = kSplit;
      nd.K[i - 1] = dk[i - 1];
    } else {
      nd.C[i - 1] = nd.C[i - 2];
      nd.D[i - 1] = kFewer;
      nd.K[i - 1] = 0;
    }
  }
  nd.costed = true;
}

// a primitive's box, centroid and index
struct Prim {
  float lo[3], hi[3], c[3];
  uint32_t id;
};

struct Bins {
  uint32_t count[3][kBins];
  Box box[3][kBins];
  void init() {
    for (int a = 0; a < 3; a++)
      for (int i = 0; i < kBins; i++) {
        count[a][i] = 0;
        box[a][i].init();
      }
  }
  void merge(const Bins& o) {
    for (int a = 0; a < 3; a++)
      for (int i = 0; i < kBins; i++) {
        count[a][i] += o.count[a][i];
        box[a][i].add(o.box[a][i]);
      }
  }
};

class Builder {
 public:
  Builder(const PrimBox* boxes, const float* cent, size_t max_leaf, unsigned threads)
      : boxes_(boxes), cent_(cent), max_leaf_(std::max<size_t>(1, std::min<size_t>(max_leaf, 8))),
        threads_(std::max(1u, threads)) {}

  // the primitives, permuted in place by the splits so that a range's
  // records are contiguous
  std::vector<Prim> prims;

  // the records and the root's bounds
  void init_prims(uint32_t n, Range& root) {
    prims.resize(n);
    unsigned const parts = n >= kParallelBins ? threads_ : 1;
    std::vector<Box> box(parts), cbox(parts);
    auto fill = [&](uint32_t b, uint32_t e, unsigned t) {
      box[t].init();
      cbox[t].init();
      for (uint32_t i = b; i < e; i++) {
        Prim& q = prims[i];
        for (int k = 0; k < 3; k++) {
          q.lo[k] = boxes_[i].inf[k];
          q.hi[k] = boxes_[i].sup[k];
          q.c[k] = cent_[3 * size_t(i) + k];
        }
        q.id = i;
        add_prim(box[t], q);
        add_cent(cbox[t], q);
      }
    };
    std::vector<std::thread> ts;
    uint32_t const chunk = (n + parts - 1) / parts;
    for (unsigned t = 0; t < parts; t++) {
      uint32_t const b = t * chunk, e = std::min(n, b + chunk);
      if (b >= e) {
        box[t].init();
        cbox[t].init();
      } else if (parts == 1) {
        fill(b, e, t);
      } else {
        ts.emplace_back(fill, b, e, t);
      }
    }
    for (auto& t : ts) t.join();
    root = Range{0, n, Box{}, Box{}};
    root.box.init();
    root.cbox.init();
    for (unsigned t = 0; t < parts; t++) {
      root.box.add(box[t]);
      root.cbox.add(cbox[t]);
    }
  }
  static void add_prim(Box& b, const Prim& q) {
    for (int k = 0; k < 3; k++) {
      b.lo[k] = std::min(b.lo[k], q.lo[k]);
      b.hi[k] = std::max(b.hi[k], q.hi[k]);
    }
  }
  static void add_cent(Box& b, const Prim& q) {
    for (int k = 0; k < 3; k++) {
      b.lo[k] = std::min(b.lo[k], q.c[k]);
      b.hi[k] = std::max(b.hi[k], q.c[k]);
    }
  }

  // Binary split of r by the binned surface-area cost (r holds at least 2
  // primitives).  par: bin on all threads (the large ranges at the top).
  void split(const Range& r, Range& left, Range& right, bool par) {
    uint32_t const n = r.size();
    if (n <= kSmall) {
      split_small(r, left, right);
      return;
    }
    // bins on the axis of the largest centroid extent
    float scale[3] = {0.f, 0.f, 0.f};
    int axis = 0;
    for (int k = 1; k < 3; k++)
      if (r.cbox.hi[k] - r.cbox.lo[k] > r.cbox.hi[axis] - r.cbox.lo[axis]) axis = k;
    float const ext = r.cbox.hi[axis] - r.cbox.lo[axis];
    scale[axis] = ext > 0.f ? float(kBins) / ext : 0.f;
    auto bin_of = [&](const Prim& p, int k) {
      int const i = int((p.c[k] - r.cbox.lo[k]) * scale[k]);
      return std::min(kBins - 1, std::max(0, i));
    };
    auto fill = [&](size_t b, size_t e, Bins& B) {
      for (size_t i = b; i < e; i++) {
        const Prim& p = prims[i];
        for (int k = 0; k < 3; k++) {
          if (scale[k] == 0.f) continue;
          int const j = bin_of(p, k);
          B.count[k][j]++;
          add_prim(B.box[k][j], p);
        }
      }
    };
    Bins bins;
    bins.init();
    unsigned const parts = par ? threads_ : 1;
    if (parts > 1) {
      std::vector<Bins> part(parts);
      std::vector<std::thread> ts;
      size_t const chunk = (n + parts - 1) / parts;
      for (unsigned t = 0; t < parts; t++) {
        size_t const b = r.b + t * chunk, e = std::min<size_t>(r.e, b + chunk);
        part[t].init();
        if (b < e) ts.emplace_back([&, b, e, t] { fill(b, e, part[t]); });
      }
      for (auto& t : ts) t.join();
      for (const Bins& B : part) bins.merge(B);
    } else {
      fill(r.b, r.e, bins);
    }
    // the cheapest plane
    double best = 1e300;
    int best_k = -1, best_j = -1;
    for (int k = 0; k < 3; k++) {
      if (scale[k] == 0.f) continue;
      double right_area[kBins];
      uint32_t right_count[kBins];
      Box acc;
      acc.init();
      uint32_t cnt = 0;
      for (int j = kBins - 1; j > 0; j--) {
        acc.add(bins.box[k][j]);
        cnt += bins.count[k][j];
        right_area[j] = acc.area();
        right_count[j] = cnt;
      }
      acc.init();
      cnt = 0;
      for (int j = 0; j < kBins - 1; j++) {
        acc.add(bins.box[k][j]);
        cnt += bins.count[k][j];
        if (cnt == 0 || right_count[j + 1] == 0) continue;
        double const cost = acc.area() * cnt + right_area[j + 1] * right_count[j + 1];
        if (cost < best) {
          best = cost;
          best_k = k;
          best_j = j;
        }
      }
    }
    left = Range{r.b, r.b, Box{}, Box{}};
    right = Range{r.e, r.e, Box{}, Box{}};
    left.box.init();
    left.cbox.init();
    right.box.init();
    right.cbox.init();
    Prim* const first = prims.data() + r.b;
    if (best_k < 0) {
      // every centroid in one point: halves in their present order
      uint32_t const mid = r.b + n / 2;
      left.e = right.b = mid;
      for (uint32_t i = r.b; i < r.e; i++) {
        Range& side = i < mid ? left : right;
        add_prim(side.box, prims[i]);
        add_cent(side.cbox, prims[i]);
      }
      return;
    }
    for (int j = 0; j < kBins; j++) (j <= best_j ? left : right).box.add(bins.box[best_k][j]);
    // partition, with each side's centroid bounds
    Prim* lo = first;
    Prim* hi = first + n;
    while (true) {
      while (lo < hi && bin_of(*lo, best_k) <= best_j) add_cent(left.cbox, *lo++);
      while (lo < hi && bin_of(*(hi - 1), best_k) > best_j) add_cent(right.cbox, *--hi);
      if (lo >= hi) break;
      std::swap(*lo, *(hi - 1));
    }
    left.e = right.b = r.b + uint32_t(lo - first);
  }

  // A small range: the exact surface-area cost of every split of its
  // primitives sorted by centroid, on each axis (no bins: their fixed cost
  // dominates near the leaves).
  void split_small(const Range& r, Range& left, Range& right) {
    uint32_t const n = r.size();
    Prim* const first = prims.data() + r.b;
    double best = 1e300;
    uint32_t best_at = n / 2;
    Prim sorted[kSmall], keep[kSmall];
    double right_area[kSmall];
    for (int k = 0; k < 3; k++) {
      std::copy(first, first + n, sorted);
      // insertion sort by centroid (stable: equal centroids keep their order)
      for (uint32_t i = 1; i < n; i++) {
        Prim const x = sorted[i];
        uint32_t j = i;
        for (; j > 0 && sorted[j - 1].c[k] > x.c[k]; j--) sorted[j] = sorted[j - 1];
        sorted[j] = x;
      }
      Box acc;
      acc.init();
      for (uint32_t i = n; i-- > 1;) {
        add_prim(acc, sorted[i]);
        right_area[i] = acc.area();
      }
      acc.init();
      bool better = false;
      for (uint32_t i = 1; i < n; i++) {
        add_prim(acc, sorted[i - 1]);
        double const cost = acc.area() * i + right_area[i] * (n - i);
        if (cost < best) {
          best = cost;
          best_at = i;
          better = true;
        }
      }
      if (better) std::copy(sorted, sorted + n, keep);
    }
    if (best < 1e300) std::copy(keep, keep + n, first);
    left = Range{r.b, r.b + best_at, Box{}, Box{}};
    right = Range{r.b + best_at, r.e, Box{}, Box{}};
    left.box.init();
    left.cbox.init();
    right.box.init();
    right.cbox.init();
    for (uint32_t i = 0; i < n; i++) {
      Range& side = i < best_at ? left : right;
      add_prim(side.box, first[i]);
      add_cent(side.cbox, first[i]);
    }
  }

  static constexpr uint32_t kParallelBins = 1u << 16;
  static constexpr uint32_t kSmall = 24;

  size_t max_leaf() const { return max_leaf_; }
  unsigned threads() const { return threads_; }

 private:
  const PrimBox* boxes_;
  const float* cent_;
  size_t max_leaf_;
  unsigned threads_;
};

// Subtrees of more than kSpawn primitives go to the queue.
constexpr uint32_t kSpawn = 1u << 10;

// A worker's nodes: fixed chunks, so a node stays in place while more are
// added (a queued subtree fills in its parent's slot) and lookups are cheap.
class NodeStore {
 public:
  static constexpr uint32_t kChunkBits = 12;
  uint32_t size() const { return n_; }
  BNode* add() {
    if ((n_ >> kChunkBits) == chunks_.size()) chunks_.emplace_back(new BNode[size_t(1) << kChunkBits]);
    BNode* nd = &chunks_[n_ >> kChunkBits][n_ & ((1u << kChunkBits) - 1)];
    n_++;
    return nd;
  }
  const BNode& operator[](uint32_t i) const { return chunks_[i >> kChunkBits][i & ((1u << kChunkBits) - 1)]; }
  BNode& at(uint32_t i) { return chunks_[i >> kChunkBits][i & ((1u << kChunkBits) - 1)]; }

 private:
  std::vector<std::unique_ptr<BNode[]>> chunks_;
  uint32_t n_ = 0;
};

class Pool {
 public:
  Pool(Builder& B, unsigned workers) : B_(B), nodes_(workers) {}

  // The tree over r; returns its root's reference.  A worker that fails
  // (no memory, no thread) stops taking subtrees; the failure is rethrown
  // here once all workers have returned.
  uint32_t run(const Range& r) {
    uint32_t root = 0;
    push(Task{r, nullptr, &root});
    std::vector<std::thread> ts;
    try {
      for (unsigned w = 1; w < nodes_.size(); w++) ts.emplace_back([this, w] { work(w); });
    } catch (...) {
      // fewer workers: the ones started and this thread finish the queue
    }
    work(0);
    for (auto& t : ts) t.join();
    if (failed_) std::rethrow_exception(failure_);
    return root;
  }

  const BNode& node(uint32_t ref) const { return nodes_[ref >> kLocalBits][ref & ((1u << kLocalBits) - 1)]; }

 private:
  struct Task {
    Range r;
    BNode* parent;  // whose kid the subtree's root becomes (null: the root)
    uint32_t* slot;
  };

  void push(const Task& t) {
    std::lock_guard<std::mutex> g(mu_);
    queue_.push_back(t);
    pending_++;
    cv_.notify_one();
  }

  void work(unsigned w) {
    while (true) {
      Task t;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return !queue_.empty() || pending_ == 0; });
        if (queue_.empty()) return;
        t = queue_.front();
        queue_.pop_front();
      }
      if (!failed_) {
        try {
          *t.slot = build(t.r, w);
        } catch (...) {
          std::lock_guard<std::mutex> g(mu_);
          if (!failed_) failure_ = std::current_exception();
          failed_ = true;
        }
      }
      std::lock_guard<std::mutex> g(mu_);
      if (--pending_ == 0) cv_.notify_all();
    }
  }

  // the binary subtree over r in worker w's nodes, costed unless a child
  // went to the queue (cost_pending then costs it)
  uint32_t build(const Range& r, unsigned w) {
    NodeStore& mine = nodes_[w];
    uint32_t const ref = (uint32_t(w) << kLocalBits) | mine.size();
    BNode* nd = mine.add();
    *nd = BNode{};
    nd->box = r.box;
    nd->b = r.b;
    nd->e = r.e;
    if (r.size() == 1) {
      nd->leaf = true;
      dp_cost(*nd, nullptr, nullptr, B_.max_leaf());
      return ref;
    }
    Range kids[2];
    B_.split(r, kids[0], kids[1], B_.threads() > 1 && r.size() > Builder::kParallelBins);
    bool queued = false;
    for (int c = 0; c < 2; c++) {
      if (kids[c].size() > kSpawn) {
        push(Task{kids[c], nd, &nd->kid[c]});
        queued = true;
      } else {
        nd->kid[c] = build(kids[c], w);
      }
    }
    if (!queued) dp_cost(*nd, &node(nd->kid[0]), &node(nd->kid[1]), B_.max_leaf());
    return ref;
  }

 public:
  // Costs the nodes whose children were built by other workers (after run).
  void cost_pending(uint32_t ref) {
    BNode& nd = node_mut(ref);
    if (nd.costed) return;
    cost_pending(nd.kid[0]);
    cost_pending(nd.kid[1]);
    dp_cost(nd, &node(nd.kid[0]), &node(nd.kid[1]), B_.max_leaf());
  }

 private:
  BNode& node_mut(uint32_t ref) { return nodes_[ref >> kLocalBits].at(ref & ((1u << kLocalBits) - 1)); }

  Builder& B_;
  std::vector<NodeStore> nodes_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<Task> queue_;
  size_t pending_ = 0;
  std::atomic<bool> failed_{false};
  std::exception_ptr failure_;
};

}  // namespace

void build_sah_bvh(uint32_t n, const PrimBox* boxes, const float* centroids, RefBvh& out, size_t max_leaf) {
  out.nodes.clear();
  out.bbs.clear();
  out.prim_idxs.clear();
  out.n_nodes = out.n_interior = 0;
  if (n == 0) return;
  unsigned const hw = std::max(1u, std::thread::hardware_concurrency());
  unsigned const workers = n > kSpawn ? std::min(hw, 64u) : 1u;
  Builder B(boxes, centroids, max_leaf, workers);
  Range root;
  B.init_prims(n, root);
  Pool P(B, workers);
  uint32_t const root_ref = P.run(root);
  P.cost_pending(root_ref);
  // the wide roots a binary subtree becomes with i of them (its decisions)
  std::vector<uint32_t> roots;
  auto roots_of = [&](auto& self, uint32_t ref, int i) -> void {
    const BNode& nd = P.node(ref);
    uint8_t const d = nd.D[i - 1];
    if (d == kFewer) {
      self(self, ref, i - 1);
    } else if (d == kSplit) {
      self(self, nd.kid[0], nd.K[i - 1]);
      self(self, nd.kid[1], i - nd.K[i - 1]);
    } else {
      roots.push_back(ref);
    }
  };
  // breadth-first numbering in the reference's layout: an interior node's
  // children are consecutive nodes, a leaf's primitives consecutive entries
  // of prim_idxs, and a record of child boxes holds its unused slots as
  // empty boxes (cg.hpp:700-727).  The numbering on this thread, the
  // records on all.
  // A wide node is a binary node that is one root: a leaf of its
  // primitives (kOneLeaf) or a wide node whose children are the roots its
  // two children become with K[0] and 8 - K[0] of them (kOneNode).
  std::vector<uint32_t> order;
  std::vector<uint32_t> at;   // per node in order: its first child, or its first primitive
  std::vector<uint32_t> rec;  // per node in order: its record of child boxes
  std::vector<uint8_t> nkid;  // per node in order: its children
  order.push_back(root_ref);
  uint32_t n_rec = 0, n_prim = 0;
  for (size_t h = 0; h < order.size(); h++) {
    const BNode& nd = P.node(order[h]);
    if (nd.D[0] == kOneLeaf) {
      at.push_back(n_prim);
      rec.push_back(0xFFFFFFFFu);
      nkid.push_back(0);
      n_prim += nd.e - nd.b;
      continue;
    }
    roots.clear();
    roots_of(roots_of, nd.kid[0], nd.K[0]);
    roots_of(roots_of, nd.kid[1], 8 - nd.K[0]);
    at.push_back(uint32_t(order.size()));
    rec.push_back(n_rec++);
    nkid.push_back(uint8_t(roots.size()));
    order.insert(order.end(), roots.begin(), roots.end());
  }
  size_t const nn = order.size();
  out.nodes.resize(2 * nn);
  out.bbs.resize(48 * size_t(n_rec));
  out.prim_idxs.resize(n_prim);
  auto fill = [&](size_t q0, size_t q1) {
    for (size_t q = q0; q < q1; q++) {
      const BNode& nd = P.node(order[q]);
      if (nkid[q] == 0) {
        out.nodes[2 * q] = 0xFFFFFFFFu;
        out.nodes[2 * q + 1] = (at[q] << 4) | ((nd.e - nd.b - 1) << 1) | 1u;
        for (uint32_t i = nd.b; i < nd.e; i++) out.prim_idxs[at[q] + (i - nd.b)] = B.prims[i].id;
        continue;
      }
      float* bb = out.bbs.data() + 48 * size_t(rec[q]);
      for (int c = 0; c < 8; c++) {
        const Box* kb = c < nkid[q] ? &P.node(order[at[q] + c]).box : nullptr;
        for (int k = 0; k < 3; k++) {
          bb[k * 8 + c] = kb ? kb->lo[k] : 1e30f;
          bb[24 + k * 8 + c] = kb ? kb->hi[k] : -1e30f;
        }
      }
      out.nodes[2 * q] = rec[q];
      out.nodes[2 * q + 1] = (at[q] << 4) | (uint32_t(nkid[q] - 1) << 1);
    }
  };
  if (workers > 1) {
    std::vector<std::thread> ts;
    size_t const chunk = (nn + workers - 1) / workers;
    for (unsigned t = 0; t < workers; t++) {
      size_t const q0 = t * chunk, q1 = std::min(nn, q0 + chunk);
      if (q0 < q1) ts.emplace_back(fill, q0, q1);
    }
    for (auto& t : ts) t.join();
  } else {
    fill(0, nn);
  }
  out.n_interior = n_rec;
  out.n_nodes = uint32_t(nn);
}

}  // namespace lgpu
