// lgpu_layout.cpp — host-side scene layout for the device.
//
// 1. build_ref_bvh restates the reference's wide BVH builder (bvh::build,
//    cg.hpp:632-749) so hosts that do not carry the reference's
//    trimeshdata can produce the identical tree: 8 bins along the longest
//    axis of the node box by triangle centroid, at most 4 primitives per
//    leaf, a full bin spread evenly over 8 children, breadth-first
//    flattening.  It also reproduces the builder's record numbering: the
//    bbs vector is first resized to n_interior and then appended to, so
//    child-box records start at index n_interior (cg.hpp:689-690, 718-722).
// 2. make_layout re-lays every mesh BVH into WideNodes (child boxes as SoA
//    rows, leaf children encoded in the parent), gathers the leaf triangles
//    in traversal order, and builds an instance-level BVH over the objects'
//    world boxes with the same builder.
#include "lgpu_layout.h"

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstring>
#include <thread>
#include <memory>
#include <queue>

namespace lgpu {

namespace {

// nl::min / nl::max (numli.hpp:60-61)
inline float nl_min(float a, float b) { return a <= b ? a : b; }
inline float nl_max(float a, float b) { return a >= b ? a : b; }

inline void box_init(PrimBox& b) {
  for (int i = 0; i < 3; i++) {
    b.inf[i] = 1e30f;
    b.sup[i] = -1e30f;
  }
}
// aabb::operator+= (cg.hpp:526-530)
inline void box_add(PrimBox& a, const PrimBox& b) {
  for (int i = 0; i < 3; i++) {
    a.inf[i] = nl_min(a.inf[i], b.inf[i]);
    a.sup[i] = nl_max(a.sup[i], b.sup[i]);
  }
}

struct BuildNode {
  PrimBox bb;
  BuildNode* children[8] = {};
  std::vector<uint32_t> prims;
  bool leaf = false;
  BuildNode(const PrimBox& b, std::vector<uint32_t> p) : bb(b), prims(std::move(p)) {}
  ~BuildNode() {
    for (BuildNode* c : children) delete c;
  }
};

constexpr size_t kPrimPerLeaf = 4;  // PRIM_PER_LEAF, cg.hpp:568 (meshes)

struct Builder {
  const PrimBox* boxes;
  const float* cent;
  size_t max_leaf;
  uint32_t n_nodes = 0, n_interior = 0;

  // bvh::splitbuildnode (cg.hpp:632-683)
  void split(BuildNode* node) {
    n_nodes++;
    if (node->prims.size() <= max_leaf) {
      node->leaf = true;
      return;
    }
    n_interior++;
    float l[3];
    for (int i = 0; i < 3; i++) l[i] = node->bb.sup[i] - node->bb.inf[i];
    int ax = 0;
    if (l[1] > l[0]) ax = 1;
    if (l[2] > l[1] && l[2] > l[0]) ax = 2;
    std::vector<uint32_t> child[8];
    for (uint32_t e : node->prims) {
      float const c = cent[3 * size_t(e) + ax];
      float const x = 8.f * (c - node->bb.inf[ax]) / l[ax];
      int b = (x >= -1.f && x < 8.f) ? int(x) : (x >= 8.f ? 7 : 0);
      b = std::min(7, std::max(0, b));
      child[b].push_back(e);
    }
    size_t const n = node->prims.size();
    for (int bin = 0; bin < 8; bin++) {
      if (child[bin].size() != n) continue;
      std::vector<uint32_t> temp = std::move(child[bin]);
      child[bin].clear();
      size_t const chunk = (n + 7) / 8;
      for (int b = 0; b < 8; b++) {
        size_t const start = b * chunk;
        size_t const end = std::min(start + chunk, n);
        if (start < end) child[b].assign(temp.begin() + start, temp.begin() + end);
      }
      break;
    }
    for (int bin = 0; bin < 8; bin++) {
      if (child[bin].empty()) continue;
      PrimBox cb;
      box_init(cb);
      for (uint32_t idx : child[bin]) box_add(cb, boxes[idx]);
      node->children[bin] = new BuildNode(cb, child[bin]);
      split(node->children[bin]);
    }
  }
};

}  // namespace

void build_ref_bvh(uint32_t n, const PrimBox* boxes, const float* centroids, RefBvh& out,
                   size_t max_leaf) {
  out = RefBvh{};
  if (n == 0) return;
  PrimBox bb;
  box_init(bb);
  std::vector<uint32_t> all(n);
  for (uint32_t i = 0; i < n; i++) {
    box_add(bb, boxes[i]);
    all[i] = i;
  }
  std::unique_ptr<BuildNode> root(new BuildNode(bb, std::move(all)));
  Builder B{boxes, centroids, max_leaf};
  B.split(root.get());
  out.n_nodes = B.n_nodes;
  out.n_interior = B.n_interior;
  // bvh::convertbuildnodes (cg.hpp:687-728)
  out.nodes.assign(2 * size_t(B.n_nodes), 0u);
  out.bbs.assign(48 * size_t(B.n_interior), 0.f);  // resize(n_interior) then append
  std::queue<std::pair<BuildNode*, uint32_t>> q;
  q.push({root.get(), 0});
  uint32_t next_free = 1;
  while (!q.empty()) {
    auto [node, idx] = q.front();
    q.pop();
    if (node->leaf) {
      uint32_t const prim_idx = uint32_t(out.prim_idxs.size());
      uint32_t const count = uint32_t(node->prims.size());
      for (uint32_t p : node->prims) out.prim_idxs.push_back(p);
      out.nodes[2 * size_t(idx)] = 0xFFFFFFFFu;
      out.nodes[2 * size_t(idx) + 1] = (prim_idx << 4) | ((count - 1) << 1) | 1u;
    } else {
      uint32_t const first = next_free;
      uint32_t nc = 0;
      PrimBox cb[8];
      for (int i = 0; i < 8; i++) box_init(cb[i]);
      for (int i = 0; i < 8; i++) {
        if (node->children[i]) {
          cb[nc] = node->children[i]->bb;
          q.push({node->children[i], next_free + nc});
          nc++;
        }
      }
      next_free += nc;
      uint32_t const bbs_idx = uint32_t(out.bbs.size() / 48);
      for (int a = 0; a < 3; a++)
        for (int c = 0; c < 8; c++) out.bbs.push_back(cb[c].inf[a]);
      for (int a = 0; a < 3; a++)
        for (int c = 0; c < 8; c++) out.bbs.push_back(cb[c].sup[a]);
      out.nodes[2 * size_t(idx)] = bbs_idx;
      out.nodes[2 * size_t(idx) + 1] = (first << 4) | ((nc - 1) << 1);
    }
  }
}

void triangle_prims(const float* V, const uint32_t* F, uint32_t f_stride, uint32_t n_faces,
                    std::vector<PrimBox>& boxes, std::vector<float>& centroids) {
  boxes.resize(n_faces);
  centroids.resize(3 * size_t(n_faces));
  for (uint32_t f = 0; f < n_faces; f++) {
    const uint32_t* t = F + size_t(f) * f_stride;
    PrimBox& b = boxes[f];
    box_init(b);
    for (int k = 0; k < 3; k++) {
      const float* v = V + 3 * size_t(t[k]);
      for (int i = 0; i < 3; i++) {
        b.inf[i] = nl_min(b.inf[i], v[i]);
        b.sup[i] = nl_max(b.sup[i], v[i]);
      }
    }
    for (int i = 0; i < 3; i++) {
      const float a = V[3 * size_t(t[0]) + i], bb = V[3 * size_t(t[1]) + i],
                  c = V[3 * size_t(t[2]) + i];
      centroids[3 * size_t(f) + i] = (a + bb + c) / 3.f;
    }
  }
}

namespace {

struct RefView {
  uint32_t n_nodes, n_bbs, n_prims;
  const uint32_t* nodes;
  const float* bbs;
  const uint32_t* prims;
};

inline bool ref_leaf(uint32_t data) { return (data & 1u) != 0; }
inline uint32_t ref_idx(uint32_t data) { return (data & 0xFFFFFFF0u) >> 4; }
inline uint32_t ref_count(uint32_t data) { return ((data & 0xEu) >> 1) + 1; }

// Runs fn(begin, end) over [0, n) on up to hardware_concurrency threads
// (one for small n).
template <class F>
void parallel_for(size_t n, F fn) {
  size_t const grain = 1 << 15;
  size_t nt = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), (n + grain - 1) / grain);
  if (nt <= 1) {
    fn(size_t(0), n);
    return;
  }
  std::vector<std::thread> ts;
  size_t const chunk = (n + nt - 1) / nt;
  for (size_t t = 0; t < nt; t++) {
    size_t const b = t * chunk, e = std::min(n, b + chunk);
    if (b < e) ts.emplace_back([=] { fn(b, e); });
  }
  for (auto& t : ts) t.join();
}

// The first pass of the relayout of a reference-format wide BVH: validates
// its nodes and gives every reference node q its child reference
// childref[q] (interior: node_base + its rank among the interior nodes;
// leaf: kLeafBit | (count-1) << 28 | slot_base + first primitive
// position).  Returns the number of interior nodes, the root reference and
// the stack bound.
bool relayout_meta(const RefView& R, uint32_t node_base, uint32_t slot_base, uint32_t* childref,
                   uint32_t& n_int_out, uint32_t& root_ref, uint32_t& max_stack, std::string& err) {
  if (R.n_nodes == 0) {
    err = "BVH has no nodes";
    return false;
  }
  uint32_t n_int = 0;
  for (uint32_t q = 0; q < R.n_nodes; q++) {
    uint32_t const d = R.nodes[2 * size_t(q) + 1];
    if (!ref_leaf(d)) {
      uint32_t const bbi = R.nodes[2 * size_t(q)];
      uint32_t const first = ref_idx(d), cnt = ref_count(d);
      if (bbi >= R.n_bbs || size_t(first) + cnt > R.n_nodes || first <= q) {
        err = "malformed BVH node";
        return false;
      }
      childref[q] = node_base + n_int++;
      continue;
    }
    uint32_t const start = ref_idx(d), cnt = ref_count(d);
    if (size_t(start) + cnt > R.n_prims) {
      err = "BVH leaf primitive range out of bounds";
      return false;
    }
    if (size_t(slot_base) + start + cnt > size_t(kMaxSlots)) {
      err = "too many leaf primitives for the device layout";
      return false;
    }
    childref[q] = kLeafBit | ((cnt - 1) << 28) | (slot_base + start);
  }
  if (size_t(node_base) + n_int >= size_t(kLeafBit)) {
    err = "too many BVH nodes";
    return false;
  }
  // entries the DFS stack can hold below each node (all children pushed),
  // children first: breadth-first indices grow downwards
  std::vector<uint32_t> bound(R.n_nodes, 0);
  for (uint32_t r = R.n_nodes; r-- > 0;) {
    uint32_t const d = R.nodes[2 * size_t(r) + 1];
    if (ref_leaf(d)) continue;
    uint32_t const first = ref_idx(d), cnt = ref_count(d);
    uint32_t deepest = 0;
    for (uint32_t c = 0; c < cnt; c++) deepest = std::max(deepest, bound[first + c]);
    bound[r] = (cnt - 1) + deepest;
  }
  n_int_out = n_int;
  root_ref = childref[0];
  max_stack = 1 + bound[0];
  return true;
}

// The second pass on the host: the WideNode of every interior node, from
// its record of child boxes and its children's references (the device
// builds the same nodes with lgpu::build_mesh_layout).
void relayout_fill(const RefView& R, const uint32_t* childref, uint32_t node_base, WideNode* nodes) {
  parallel_for(R.n_nodes, [&](size_t r0, size_t r1) {
    for (size_t r = r0; r < r1; r++) {
      uint32_t const d = R.nodes[2 * r + 1];
      if (ref_leaf(d)) continue;
      const float* bb = R.bbs + 48 * size_t(R.nodes[2 * r]);
      uint32_t const first = ref_idx(d), cnt = ref_count(d);
      WideNode& wn = nodes[childref[r] - node_base];
      for (int c = 0; c < 8; c++) {
        if (uint32_t(c) < cnt) {
          wn.lox[c] = bb[0 * 8 + c];
          wn.loy[c] = bb[1 * 8 + c];
          wn.loz[c] = bb[2 * 8 + c];
          wn.hix[c] = bb[3 * 8 + c];
          wn.hiy[c] = bb[4 * 8 + c];
          wn.hiz[c] = bb[5 * 8 + c];
          wn.child[c] = childref[first + c];
        } else {
          wn.lox[c] = wn.loy[c] = wn.loz[c] = 1e30f;
          wn.hix[c] = wn.hiy[c] = wn.hiz[c] = -1e30f;
          wn.child[c] = kEmptyChild;
        }
      }
    }
  });
}

// Re-lays a reference-format wide BVH into WideNodes appended to `nodes`
// (node indices continue from node_base, the index of nodes[0]).  Leaf
// children point at slot_base + (first primitive position).  Returns the
// root reference through root_ref and the stack bound through max_stack.
bool relayout(const RefView& R, uint32_t node_base, uint32_t slot_base, BigVector<WideNode>& nodes,
              uint32_t& root_ref, uint32_t& max_stack, std::string& err) {
  std::vector<uint32_t> childref(R.n_nodes);
  uint32_t n_int = 0;
  uint32_t const first = node_base + uint32_t(nodes.size());
  if (!relayout_meta(R, first, slot_base, childref.data(), n_int, root_ref, max_stack, err)) return false;
  size_t const at = nodes.size();
  nodes.resize(at + n_int);
  relayout_fill(R, childref.data(), first, nodes.data() + at);
  return true;
}

bool finite3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

}  // namespace

// The material table of a scene (validated), as the kernels read it.
int make_materials(const lgpu_scene& sc, std::vector<DevMaterial>& mats, std::string& err) {
  mats.clear();
  auto spec_ok = [&](int32_t s) { return s >= 0 && uint32_t(s) < sc.n_spectra; };
  for (uint32_t i = 0; i < sc.n_materials; i++) {
    const lgpu_material& m = sc.materials[i];
    DevMaterial d{};
    d.type = m.type;
    for (int k = 0; k < 5; k++) d.spectrum[k] = m.spectrum[k];
    d.alpha = m.alpha;
    d.p_d = m.p_d;
    d.p_spec = m.p_spec;
    d.w_r = m.w_r;
    d.w_t = m.w_t;
    d.d = m.d;
    d.specular = m.specular;
    int need = 0;
    switch (m.type) {
      case LGPU_MAT_LAMBERTIAN: need = 1; break;
      case LGPU_MAT_BLINN: need = 5; break;
      case LGPU_MAT_THINFILM: need = 2; break;
      case LGPU_MAT_MICROFACET: need = 0; break;
      case LGPU_MAT_EMITTER:
      case LGPU_MAT_DIREMITTER: need = 1; break;
      default:
        err = "unknown material type";
        return LGPU_ERR_INVALID_ARGUMENT;
    }
    for (int k = 0; k < need; k++)
      if (!spec_ok(m.spectrum[k])) {
        err = "material spectrum index out of range";
        return LGPU_ERR_INVALID_ARGUMENT;
      }
    mats.push_back(d);
  }
  return LGPU_OK;
}

int make_layout(const lgpu_scene& sc, HostLayout& L, std::string& err, DeviceLayoutWork* dev,
                const std::vector<TravTree>* trav) {
  if (dev) {
    dev->jobs.clear();
    dev->childref.clear();
    dev->mesh_nodes = dev->mesh_slots = dev->mesh_faces = 0;
  }
  // empty every array but keep its capacity
  L.objects.clear();
  L.meshes.clear();
  L.nodes.clear();
  L.tris.clear();
  L.shade.clear();
  L.spectra.clear();
  L.mats.clear();
  L.lights.clear();
  L.tlas_objects.clear();
  L.cmf.clear();
  L.tlas_root = L.max_stack = L.tlas_max_stack = 0;
  for (float& b : L.tlas_bounds) b = 0.f;
  const lgpu_spectral& sp = sc.spec;
  if (sp.n_bins < 2 || !(sp.lambda_sup > sp.lambda_inf)) {
    err = "spectral discretisation needs n_bins >= 2 and lambda_sup > lambda_inf";
    return LGPU_ERR_INVALID_ARGUMENT;
  }
  if (sp.hero_k != 4 && sp.hero_k != 8 && sp.hero_k != 16) {
    err = "hero_k must be 4, 8 or 16";
    return LGPU_ERR_UNSUPPORTED;
  }
  if (!sp.cmf_x || !sp.cmf_y || !sp.cmf_z) {
    err = "CMF tables missing";
    return LGPU_ERR_INVALID_ARGUMENT;
  }
  if (sc.cam.width == 0 || sc.cam.height == 0 || sc.cam.width * sc.cam.height > (1ull << 31)) {
    err = "camera resolution out of range";
    return LGPU_ERR_INVALID_ARGUMENT;
  }
  if (sc.n_lights == 0 || !sc.lights) {
    // sample::lights takes rng.uint64() % n (cg.hpp:1553)
    err = "the scene has no lights";
    return LGPU_ERR_INVALID_ARGUMENT;
  }
  if ((sc.n_objects && !sc.objects) || (sc.n_materials && !sc.materials) ||
      (sc.n_meshes && !sc.meshes) || (sc.n_spectra && !sc.spectra)) {
    err = "null array with a non-zero count";
    return LGPU_ERR_INVALID_ARGUMENT;
  }
  uint32_t const nb = sp.n_bins;
  L.spectra.assign(sc.spectra, sc.spectra + size_t(sc.n_spectra) * nb);
  L.cmf.resize(3 * size_t(nb));
  std::memcpy(L.cmf.data(), sp.cmf_x, nb * sizeof(float));
  std::memcpy(L.cmf.data() + nb, sp.cmf_y, nb * sizeof(float));
  std::memcpy(L.cmf.data() + 2 * nb, sp.cmf_z, nb * sizeof(float));

  auto spec_ok = [&](int32_t s) { return s >= 0 && uint32_t(s) < sc.n_spectra; };
  if (int rc = make_materials(sc, L.mats, err)) return rc;
  // lights
  for (uint32_t i = 0; i < sc.n_lights; i++) {
    const lgpu_light& l = sc.lights[i];
    if (l.type < LGPU_LIGHT_AMBIENT || l.type > LGPU_LIGHT_QUADDIR || !spec_ok(l.spectrum)) {
      err = "invalid light";
      return LGPU_ERR_INVALID_ARGUMENT;
    }
    if ((l.type == LGPU_LIGHT_SPHERE || l.type == LGPU_LIGHT_QUADDIR) && l.obj >= sc.n_objects) {
      err = "light object index out of range";
      return LGPU_ERR_INVALID_ARGUMENT;
    }
    L.lights.push_back(l);
  }
  // meshes
  for (uint32_t mi = 0; mi < sc.n_meshes; mi++) {
    const lgpu_mesh& m = sc.meshes[mi];
    if (m.n_faces == 0 || !m.V || !m.F || !m.N || !m.GN || !m.nodes || !m.bbs || !m.prim_idxs ||
        m.f_stride < 6) {
      err = "incomplete mesh " + std::to_string(mi);
      return LGPU_ERR_INVALID_ARGUMENT;
    }
    DevMesh dm{};
    dm.n_faces = m.n_faces;
    std::memcpy(dm.bounds, m.bounds, sizeof(dm.bounds));
    RefView const R{m.n_nodes, m.n_bbs, m.n_prim_idxs, m.nodes, m.bbs, m.prim_idxs};
    if (dev) {
      // the device builds this mesh's nodes, leaf triangles and shading
      // normals (and checks its face and primitive indices) from its raw
      // arrays; here only the child references and the stack bound
      DeviceMeshJob j{};
      j.mesh = mi;
      j.node_base = dev->mesh_nodes;
      j.slot_base = dev->mesh_slots;
      j.face_base = dev->mesh_faces;
      j.childref_off = dev->childref.size();
      dev->childref.resize(j.childref_off + m.n_nodes);
      if (!relayout_meta(R, j.node_base, j.slot_base, dev->childref.data() + j.childref_off, j.n_int, dm.root,
                         dm.max_stack, err)) {
        err = "mesh " + std::to_string(mi) + ": " + err;
        return LGPU_ERR_INVALID_ARGUMENT;
      }
      if (dm.max_stack > uint32_t(kStackCap)) {
        err = "mesh " + std::to_string(mi) + " BVH can need " + std::to_string(dm.max_stack) +
              " stack entries; the traversal holds " + std::to_string(kStackCap);
        return LGPU_ERR_UNSUPPORTED;
      }
      dm.node_base = j.node_base;
      dm.slot_base = j.slot_base;
      dm.face_base = j.face_base;
      dm.trav_root = dm.root;
      dev->mesh_nodes += j.n_int;
      dev->mesh_slots += m.n_prim_idxs;
      dev->mesh_faces += m.n_faces;
      dev->jobs.push_back(j);
      L.max_stack = std::max(L.max_stack, dm.max_stack);
      const TravTree* T = trav && mi < trav->size() && (*trav)[mi].n_nodes ? &(*trav)[mi] : nullptr;
      if (T) {
        // the traversal tree: its own nodes and leaf slots, the mesh's faces
        RefView const R2{T->n_nodes, T->n_bbs, T->n_prims, T->nodes, T->bbs, T->prims};
        DeviceMeshJob t{};
        t.mesh = mi;
        t.node_base = dev->mesh_nodes;
        t.slot_base = dev->mesh_slots;
        t.face_base = j.face_base;
        t.childref_off = dev->childref.size();
        t.tree = T;
        dev->childref.resize(t.childref_off + R2.n_nodes);
        uint32_t root2 = 0, stack2 = 0;
        if (!relayout_meta(R2, t.node_base, t.slot_base, dev->childref.data() + t.childref_off, t.n_int, root2,
                           stack2, err)) {
          err = "mesh " + std::to_string(mi) + " traversal tree: " + err;
          return LGPU_ERR_INVALID_ARGUMENT;
        }
        // a tree deeper than the traversal stack is dropped: the mesh's own
        // tree serves
        if (stack2 <= uint32_t(kStackCap)) {
          dm.trav_root = root2;
          dev->mesh_nodes += t.n_int;
          dev->mesh_slots += R2.n_prims;
          dev->jobs.push_back(t);
          L.max_stack = std::max(L.max_stack, stack2);
        } else {
          dev->childref.resize(t.childref_off);
        }
      }
      L.meshes.push_back(dm);
      continue;
    }
    std::atomic<bool> bad_face{false}, bad_prim{false};
    parallel_for(m.n_faces, [&](size_t f0, size_t f1) {
      for (size_t f = f0; f < f1; f++) {
        const uint32_t* t = m.F + f * m.f_stride;
        for (int k = 0; k < 3; k++)
          if (t[k] >= m.n_positions || t[3 + k] >= m.n_normals) bad_face = true;
      }
    });
    parallel_for(m.n_prim_idxs, [&](size_t s0, size_t s1) {
      for (size_t s = s0; s < s1; s++)
        if (m.prim_idxs[s] >= m.n_faces) bad_prim = true;
    });
    if (bad_face) {
      err = "face index out of range in mesh " + std::to_string(mi);
      return LGPU_ERR_INVALID_ARGUMENT;
    }
    if (bad_prim) {
      err = "BVH primitive index out of range in mesh " + std::to_string(mi);
      return LGPU_ERR_INVALID_ARGUMENT;
    }
    dm.slot_base = uint32_t(L.tris.size());
    dm.face_base = uint32_t(L.shade.size());
    dm.node_base = uint32_t(L.nodes.size());
    if (!relayout(R, 0, dm.slot_base, L.nodes, dm.root, dm.max_stack, err)) {
      err = "mesh " + std::to_string(mi) + ": " + err;
      return LGPU_ERR_INVALID_ARGUMENT;
    }
    if (dm.max_stack > uint32_t(kStackCap)) {
      err = "mesh " + std::to_string(mi) + " BVH can need " + std::to_string(dm.max_stack) +
            " stack entries; the traversal holds " + std::to_string(kStackCap);
      return LGPU_ERR_UNSUPPORTED;
    }
    L.max_stack = std::max(L.max_stack, dm.max_stack);
    // the leaf triangles of a tree whose leaves list the faces `prims`
    auto fill_tris = [&](const uint32_t* prims, size_t n_prims, TriSlot* tris) {
      parallel_for(n_prims, [&](size_t s0, size_t s1) {
        for (size_t s = s0; s < s1; s++) {
          uint32_t const f = prims[s];
          const uint32_t* t = m.F + size_t(f) * m.f_stride;
          TriSlot& ts = tris[s];
          const float* a = m.V + 3 * size_t(t[0]);
          const float* b = m.V + 3 * size_t(t[1]);
          const float* c = m.V + 3 * size_t(t[2]);
          for (int i = 0; i < 3; i++) {
            ts.v0[i] = a[i];
            ts.v1[i] = b[i];
            ts.v2[i] = c[i];
          }
          std::memcpy(&ts.v0[3], &f, 4);
          ts.v1[3] = 0.f;
          ts.v2[3] = 0.f;
        }
      });
    };
    size_t const tri0 = L.tris.size(), shade0 = L.shade.size();
    L.tris.resize(tri0 + m.n_prim_idxs);
    L.shade.resize(shade0 + m.n_faces);
    FaceShade* const shades = L.shade.data() + shade0;
    fill_tris(m.prim_idxs, m.n_prim_idxs, L.tris.data() + tri0);
    parallel_for(m.n_faces, [&](size_t f0, size_t f1) {
      for (size_t f = f0; f < f1; f++) {
        const uint32_t* t = m.F + f * m.f_stride;
        FaceShade& fs = shades[f];
        for (int i = 0; i < 3; i++) {
          fs.n0[i] = m.N[3 * size_t(t[3]) + i];
          fs.n1[i] = m.N[3 * size_t(t[4]) + i];
          fs.n2[i] = m.N[3 * size_t(t[5]) + i];
          fs.gn[i] = m.GN[3 * f + i];
        }
      }
    });
    dm.trav_root = dm.root;
    const TravTree* T = trav && mi < trav->size() && (*trav)[mi].n_nodes ? &(*trav)[mi] : nullptr;
    if (T) {
      // the traversal tree: its own nodes and leaf slots, the mesh's faces
      RefView const R2{T->n_nodes, T->n_bbs, T->n_prims, T->nodes, T->bbs, T->prims};
      size_t const nodes0 = L.nodes.size(), slot2 = L.tris.size();
      uint32_t root2 = 0, stack2 = 0;
      std::atomic<bool> bad_trav{false};
      parallel_for(R2.n_prims, [&](size_t s0, size_t s1) {
        for (size_t q = s0; q < s1; q++)
          if (R2.prims[q] >= m.n_faces) bad_trav = true;
      });
      if (bad_trav) {
        err = "traversal-tree primitive index out of range in mesh " + std::to_string(mi);
        return LGPU_ERR_INVALID_ARGUMENT;
      }
      if (!relayout(R2, 0, uint32_t(slot2), L.nodes, root2, stack2, err)) {
        err = "mesh " + std::to_string(mi) + " traversal tree: " + err;
        return LGPU_ERR_INVALID_ARGUMENT;
      }
      // a tree deeper than the traversal stack is dropped: the mesh's own
      // tree serves
      if (stack2 <= uint32_t(kStackCap)) {
        L.tris.resize(slot2 + R2.n_prims);
        fill_tris(R2.prims, R2.n_prims, L.tris.data() + slot2);
        dm.trav_root = root2;
        L.max_stack = std::max(L.max_stack, stack2);
      } else {
        L.nodes.resize(nodes0);
      }
    }
    L.meshes.push_back(dm);
  }
  // objects and their world boxes
  std::vector<PrimBox> boxes(sc.n_objects);
  std::vector<float> cents(3 * size_t(sc.n_objects));
  for (uint32_t i = 0; i < sc.n_objects; i++) {
    const lgpu_object& o = sc.objects[i];
    if (o.type < LGPU_OBJ_SPHERE || o.type > LGPU_OBJ_TRIMESH || o.mat >= sc.n_materials ||
        (o.type == LGPU_OBJ_TRIMESH && o.mesh >= sc.n_meshes)) {
      err = "invalid object " + std::to_string(i);
      return LGPU_ERR_INVALID_ARGUMENT;
    }
    DevObject d{};
    d.type = o.type;
    d.mat = o.mat;
    d.mesh = o.mesh;
    std::memcpy(d.M, o.T.M, 12 * sizeof(float));
    std::memcpy(d.M_inv, o.T.M_inv, 12 * sizeof(float));
    L.objects.push_back(d);
    float lo[3] = {-1.f, -1.f, -1.f}, hi[3] = {1.f, 1.f, 1.f};
    if (o.type == LGPU_OBJ_PLANE) lo[2] = hi[2] = 0.f;
    if (o.type == LGPU_OBJ_TRIMESH) {
      const float* b = sc.meshes[o.mesh].bounds;
      for (int k = 0; k < 3; k++) {
        lo[k] = b[k];
        hi[k] = b[3 + k];
      }
    }
    double wlo[3] = {1e300, 1e300, 1e300}, whi[3] = {-1e300, -1e300, -1e300};
    for (int c = 0; c < 8; c++) {
      double const p[3] = {(c & 1) ? hi[0] : lo[0], (c & 2) ? hi[1] : lo[1], (c & 4) ? hi[2] : lo[2]};
      for (int r = 0; r < 3; r++) {
        double const w = double(o.T.M[4 * r]) * p[0] + double(o.T.M[4 * r + 1]) * p[1] +
                         double(o.T.M[4 * r + 2]) * p[2] + double(o.T.M[4 * r + 3]);
        wlo[r] = std::min(wlo[r], w);
        whi[r] = std::max(whi[r], w);
      }
    }
    if (!finite3(o.T.M) || !finite3(o.T.M + 4) || !finite3(o.T.M + 8)) {
      err = "non-finite transform on object " + std::to_string(i);
      return LGPU_ERR_INVALID_ARGUMENT;
    }
    for (int r = 0; r < 3; r++) {
      // pad so rounding in the object's own test can never fall outside
      double const mag = std::max({std::fabs(wlo[r]), std::fabs(whi[r]), whi[r] - wlo[r]});
      double const pad = 1e-5 * mag + 1e-6;
      boxes[i].inf[r] = float(wlo[r] - pad);
      boxes[i].sup[r] = float(whi[r] + pad);
      cents[3 * size_t(i) + r] = 0.5f * (boxes[i].inf[r] + boxes[i].sup[r]);
    }
  }
  // no objects: an empty instance-BVH box that no ray enters
  for (int k = 0; k < 3; k++) {
    L.tlas_bounds[k] = 1e30f;
    L.tlas_bounds[3 + k] = -1e30f;
  }
  if (sc.n_objects > 0) {
    // one object per leaf: objects are culled by the 8-wide box test.  Only
    // the instance-BVH traversal enters it (the reference order loops over
    // the objects), so it is built with the surface-area heuristic: 9.4
    // node tests per ray instead of 12.0 with the reference's split rule on
    // the benchmark scene (frame +10.5 %, measured).  A tree whose stack
    // bound exceeds the traversal's instance stack (thousands of objects
    // can) is replaced by the reference's split rule, whose 8-way slabs
    // give shallower trees.
    size_t const nodes0 = L.nodes.size();
    for (int attempt = 0; attempt < 2; attempt++) {
      RefBvh tl;
      if (attempt == 0)
        build_sah_bvh(sc.n_objects, boxes.data(), cents.data(), tl, 1);
      else
        build_ref_bvh(sc.n_objects, boxes.data(), cents.data(), tl, 1);
      L.tlas_objects = tl.prim_idxs;
      RefView const R{tl.n_nodes, uint32_t(tl.bbs.size() / 48), uint32_t(tl.prim_idxs.size()),
                      tl.nodes.data(), tl.bbs.data(), tl.prim_idxs.data()};
      L.nodes.resize(nodes0);
      // after the meshes' nodes, wherever those are built
      if (!relayout(R, dev ? dev->mesh_nodes : 0, 0, L.nodes, L.tlas_root, L.tlas_max_stack, err)) {
        err = "instance BVH: " + err;
        return LGPU_ERR_INVALID_ARGUMENT;
      }
      if (L.tlas_max_stack <= uint32_t(kTlasStackCap)) break;
      if (attempt == 1) {
        err = "instance BVH can need " + std::to_string(L.tlas_max_stack) + " stack entries";
        return LGPU_ERR_UNSUPPORTED;
      }
    }
    PrimBox all;
    box_init(all);
    for (const PrimBox& b : boxes) box_add(all, b);
    for (int k = 0; k < 3; k++) {
      L.tlas_bounds[k] = all.inf[k];
      L.tlas_bounds[3 + k] = all.sup[k];
    }
  }
  return LGPU_OK;
}

}  // namespace lgpu
