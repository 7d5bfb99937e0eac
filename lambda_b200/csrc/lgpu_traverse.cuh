// lgpu_traverse.cuh — the instance-level traversal used by the wavefront
// kernels: one loop over instance-BVH and mesh-BVH nodes with a single
// stack, so that all lanes of a warp execute the same "pop, test, push"
// step whatever level they are at.
//
// Entering a mesh pushes a marker and the mesh root; popping the marker
// returns to world space.  A leaf of the instance BVH is consumed one object
// at a time (the rest of the leaf is pushed back), which visits objects and
// mesh nodes in exactly the order of the nested traversal in
// lgpu_intersect.cuh, so results are identical to it (and therefore to the
// reference's intersect::scene, see scene_hit).
//
// The stack keeps its first kSmemStack entries in shared memory, laid out
// entry-major (entry k of thread t at k*blockDim.x + t) so a warp's pushes
// and pops hit distinct banks; deeper entries go to a per-thread local
// array.
#pragma once

#include "lgpu_intersect.cuh"

namespace lgpu {

// The instance-BVH traversal tests boxes with a relative slack: a child is
// kept while its rounded entry distance is at most (1 + 2^-16) times its
// rounded exit (the closest hit so far included), and a popped entry is
// dropped only beyond (1 + 2^-16) times the closest hit.  A box's rounded
// entry can lie a few ulps beyond a triangle it contains (its vertex on the
// box's face), and without the slack such a triangle can be culled when a
// neighbouring one was hit first (one ray of 1.14 million in the benchmark
// scene traced with the surface-area-heuristic trees).  The slack only adds
// node tests; the reference-order traversal keeps the exact test.
constexpr float kTravSlack = 1.f + 1.f / 65536.f;

constexpr int kSmemStack = 16;
constexpr int kLocalStack = kStackCap + kTlasStackCap + 4 - kSmemStack;
constexpr uint32_t kMarker = 0xFFFFFFFEu;

struct SplitStack {
  StackEntry* sm;  // this thread's column in shared memory
  uint32_t stride;
  StackEntry* lm;  // local overflow
  int sp;
  // kTravLocalStack once an entry beyond the shared part was used (merged
  // into the thread's TravStats::flags when its work is counted)
  uint32_t spill;
  // this thread's column of the world-ray save area (9 floats, stride 128;
  // trace_step only)
  float* ws = nullptr;
  __device__ __forceinline__ StackEntry& at(int k) {
    if (k < kSmemStack) return sm[k * stride];
    spill = kTravLocalStack;
    return lm[k - kSmemStack];
  }
  // push and pop branch to a shared or a local access: through at()'s
  // reference the compiler emits generic loads and stores, which cost
  // registers (spills) and issue slots (traversal -6 % measured)
  __device__ __forceinline__ void push(StackEntry e) {
    if (sp < kSmemStack) {
      sm[sp * stride] = e;
    } else {
      spill = kTravLocalStack;
      lm[sp - kSmemStack] = e;
    }
    sp++;
  }
  __device__ __forceinline__ StackEntry pop() {
    --sp;
    if (sp < kSmemStack) return sm[sp * stride];
    return lm[sp - kSmemStack];
  }
};

constexpr int kSplitCap = kSmemStack + kLocalStack;

// push_children (lgpu_intersect.cuh) writing through a SplitStack.  With
// `sorted` false (any-hit queries, whose boolean answer does not depend on
// the visiting order) the hit children are pushed in child order.
template <bool ROWS>
__device__ __forceinline__ bool push_children_split(const WideNode& nd, const Ray& r, float t_max,
                                                    SplitStack& st, bool sorted) {
  float t[8];
  uint32_t ref[8];
  // ROWS: the row-wise test (the persistent kernels, which have the
  // registers for it); otherwise the per-child test (both give the same t)
  if (ROWS) {
    node_boxes_t(nd, r, t_max, t, kTravSlack);
#pragma unroll
    for (int c = 0; c < 8; c++) {
      ref[c] = nd.child[c];
      if (ref[c] == kEmptyChild) t[c] = 0.f;
    }
  } else {
    bool const nx = r.inv.x < 0.f, ny = r.inv.y < 0.f, nz = r.inv.z < 0.f;
#pragma unroll
    for (int c = 0; c < 8; c++) {
      ref[c] = nd.child[c];
      t[c] = (ref[c] != kEmptyChild) ? child_box_t(nd, c, r, nx, ny, nz, t_max, kTravSlack) : 0.f;
    }
  }
  int hits = 0;
#pragma unroll
  for (int c = 0; c < 8; c++) hits += (t[c] != 0.f) ? 1 : 0;
  if (st.sp + hits > kSplitCap) return false;
  if (!sorted) {
    if (st.sp + hits <= kSmemStack) {
      // as below: shared-memory stores only
      StackEntry* p = st.sm + st.sp * st.stride;
#pragma unroll
      for (int c = 0; c < 8; c++)
        if (t[c] != 0.f) {
          *p = StackEntry{ref[c], t[c]};
          p += st.stride;
        }
      st.sp += hits;
      return true;
    }
#pragma unroll
    for (int c = 0; c < 8; c++)
      if (t[c] != 0.f) st.push(StackEntry{ref[c], t[c]});
    return true;
  }
  // Far to near by a sorting network on 32-bit keys: a hit's distance bits
  // with their 3 low bits replaced by 7 - child (equal distances keep child
  // order; a miss's key, 7 - child alone, is below every hit's).  19
  // compare-exchanges of integer max/min cost fewer instructions than the
  // pairwise ranks of push_children (measured: closest-hit traversal
  // -1.4 %), and the hits are then pushed in sequence with their child
  // references read again from the node (an L1 hit) instead of kept in
  // registers.  The order can differ from the exact far-to-near order only
  // between children whose entry distances lie within 8 ulps, which changes
  // no closest distance (ties only; the reference-order traversal keeps
  // push_children's exact order).  The stored distance is the key's, at
  // most 7 ulps below the box's, so an entry is never culled early.
  uint32_t key[8];
#pragma unroll
  for (int c = 0; c < 8; c++) key[c] = (t[c] != 0.f ? (__float_as_uint(t[c]) & ~7u) : 0u) | uint32_t(7 - c);
  constexpr int kNet[19][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6}, {5, 7}, {1, 2}, {5, 6},
                               {0, 4}, {3, 7}, {1, 5}, {2, 6}, {1, 4}, {3, 6}, {2, 4}, {3, 5}, {3, 4}};
#pragma unroll
  for (int k = 0; k < 19; k++) {
    uint32_t const a = key[kNet[k][0]], b = key[kNet[k][1]];
    key[kNet[k][0]] = max(a, b);
    key[kNet[k][1]] = min(a, b);
  }
  if (st.sp + hits <= kSmemStack) {
    // every hit lands in the shared part of the stack: no per-entry choice of memory
    StackEntry* const p = st.sm + st.sp * st.stride;
#pragma unroll
    for (int j = 0; j < 8; j++)
      if (j < hits) p[j * st.stride] = StackEntry{nd.child[7 - (key[j] & 7u)], __uint_as_float(key[j] & ~7u)};
    st.sp += hits;
    return true;
  }
#pragma unroll
  for (int j = 0; j < 8; j++)
    if (j < hits) st.at(st.sp + j) = StackEntry{nd.child[7 - (key[j] & 7u)], __uint_as_float(key[j] & ~7u)};
  st.sp += hits;
  return true;
}

// Instance-BVH traversal with the same semantics as scene_hit's instance
// path (ties to the higher object index, inside-bounds meshes tested in full
// and flagged in the hit).  Returns whether a hit was accepted.
template <bool ANY>
__device__ __forceinline__ bool trace_tlas(const DevScene& S, const Ray& w, HitRec& h, uint32_t skip,
                                           SplitStack& st, TravStats& ts) {
  h.inside = false;
  if (S.n_objects == 0) return false;
  float const t0 = segment_box_entry(S.tlas_bounds, w, h.z);
  if (t0 == kFltMax) return false;
  st.sp = 0;
  st.push(StackEntry{S.tlas_root, t0});
  bool in_mesh = false, lowered = false, cur_inside = false, hit_any = false;
  Ray l = w;
  f3 mr = f3{0.f, 0.f, 0.f};
  uint32_t cur = 0;
  float zs = 0.f, cur_exit = 0.f;
  while (st.sp > 0) {
    StackEntry const e = st.pop();
    if (e.ref == kMarker) {
      in_mesh = false;
      if (lowered && h.obj != cur) h.z = zs;
      lowered = false;
      continue;
    }
    if (e.t > h.z * kTravSlack) continue;
    if (!(e.ref & kLeafBit)) {
      ts.nodes++;
      if (!push_children_split<ANY>(S.nodes[e.ref], in_mesh ? l : w, h.z, st, !ANY)) {
        ts.flags |= 1u;
        break;
      }
      continue;
    }
    uint32_t const cnt = ((e.ref >> 28) & 7u) + 1u;
    uint32_t const slot = e.ref & kSlotMask;
    if (in_mesh) {
      for (uint32_t k = 0; k < cnt; k++) {
        const TriSlot& T = S.tris[slot + k];
        ts.tris++;
        float t, b0, b1, b2;
        if (tri_test(T, l, mr, h.z, t, b0, b1, b2)) {
          h.z = t;
          h.obj = cur;
          h.face = __float_as_uint(T.v0[3]);
          h.b0 = b0;
          h.b1 = b1;
          h.b2 = b2;
          h.pl = ray_at(l, t);
          h.inside = cur_inside;
          h.exit = cur_exit;
          hit_any = true;
          if (ANY) return true;
        }
      }
      continue;
    }
    // instance leaf: the first object now, the rest of the leaf afterwards
    uint32_t const i = S.tlas_objects[slot];
    if (cnt > 1) {
      if (st.sp + 1 > kSplitCap) {
        ts.flags |= 1u;
        break;
      }
      st.push(StackEntry{kLeafBit | ((cnt - 2u) << 28) | (slot + 1u), e.t});
    }
    if (i == skip) continue;
    ts.insts++;
    const DevObject& ob = S.objects[i];
    bool const low = !ANY && h.obj != UINT32_MAX && i < h.obj;
    float const z_saved = h.z;
    if (low) h.z = prev_float(z_saved);
    Ray const li = to_local(ob, w);
    if (ob.type != LGPU_OBJ_TRIMESH) {
      float t;
      f3 x;
      bool hit;
      if (ob.type == LGPU_OBJ_SPHERE) {
        hit = sphere_test(li, h.z, t);
        if (hit) x = ray_at(li, t);
      } else {
        hit = plane_test(li, h.z, t, x);
      }
      if (hit) {
        h.z = t;
        h.obj = i;
        h.face = UINT32_MAX;
        h.pl = x;
        h.inside = false;
        hit_any = true;
        if (ANY) return true;
      } else if (low) {
        h.z = z_saved;
      }
      continue;
    }
    const DevMesh& m = S.meshes[ob.mesh];
    bool inside;
    float ex;
    float r0 = aabb_scalar(m.bounds, li, h.z, inside, ex);
    if (r0 != kFltMax && !ANY && inside) r0 = kBias;
    if (r0 == kFltMax || r0 > h.z) {
      if (low) h.z = z_saved;
      continue;
    }
    if (st.sp + 2 > kSplitCap) {
      ts.flags |= 1u;
      break;
    }
    l = li;
    mr = cross3(l.p, l.u);
    cur = i;
    cur_inside = inside;
    cur_exit = ex;
    zs = z_saved;
    lowered = low;
    in_mesh = true;
    st.push(StackEntry{kMarker, 0.f});
    st.push(StackEntry{m.trav_root, r0});
  }
  return hit_any;
}

// trace_tlas as a resumable state machine: trace_begin sets up a ray,
// trace_step processes one stack entry.  The persistent trace kernels call
// trace_step in a loop shared by the whole warp and give a lane a new ray
// as soon as its ray is finished, so lanes do not idle while the longest ray
// of their warp completes.
// Besides the ray, a query has a mode (`any`: stop at the first hit, as
// shadow rays do), an object to skip and an index limit (objects with a
// higher or equal index are ignored), and counts the meshes whose bounds
// contain the ray origin (n_inside).
// `w` is the ray of the current level: the world ray, or the mesh-local ray
// while a mesh is entered, when the world ray waits in shared memory
// (SplitStack::ws) until the mesh's end marker.  One ray in registers
// instead of two lets the closest-hit kernel run 6 blocks per SM without
// spills (traversal -4 % measured).
struct TraceState {
  Ray w;
  f3 mr;
  HitRec h;
  uint32_t skip, ilimit, cur;
  float zs, cur_exit;
  uint32_t n_inside;
  bool any, in_mesh, lowered, cur_inside, hit_any;
};

__device__ __forceinline__ void trace_begin(const DevScene& S, TraceState& t, SplitStack& st) {
  t.h.inside = false;
  t.in_mesh = t.lowered = t.cur_inside = t.hit_any = false;
  t.cur = 0;
  t.n_inside = 0;
  t.zs = t.cur_exit = 0.f;
  st.sp = 0;
  if (S.n_objects == 0) return;  // no instance BVH: every ray misses
  float const t0 = segment_box_entry(S.tlas_bounds, t.w, t.h.z);
  if (t0 != kFltMax) st.push(StackEntry{S.tlas_root, t0});
}

// One step of trace_tlas; returns true when the ray is finished (stack
// empty, or an any-hit query found a hit).  ANY fixes the mode at compile
// time; otherwise t.any selects it.
template <bool ANY>
__device__ __forceinline__ bool trace_step(const DevScene& S, TraceState& t, SplitStack& st,
                                           TravStats& ts) {
  if (st.sp == 0) return true;
  bool const any = ANY || t.any;
  StackEntry const e = st.pop();
  HitRec& h = t.h;
  if (e.ref == kMarker) {
    t.in_mesh = false;
    if (t.lowered && h.obj != t.cur) h.z = t.zs;
    t.lowered = false;
    t.w.p = f3{st.ws[0], st.ws[128], st.ws[2 * 128]};
    t.w.u = f3{st.ws[3 * 128], st.ws[4 * 128], st.ws[5 * 128]};
    t.w.inv = f3{st.ws[6 * 128], st.ws[7 * 128], st.ws[8 * 128]};
    return st.sp == 0;
  }
  if (e.t > h.z * kTravSlack) return st.sp == 0;
  if (!(e.ref & kLeafBit)) {
    ts.nodes++;
    // children near to far, except in the shadow kernel: its answer does not
    // depend on the order, and sorting costs it more than it saves.  (The
    // closest-hit kernel's own any-hit queries are faster sorted.)
    if (!push_children_split<true>(S.nodes[e.ref], t.w, h.z, st, !ANY)) {
      ts.flags |= 1u;
      return true;
    }
    return st.sp == 0;
  }
  uint32_t const cnt = ((e.ref >> 28) & 7u) + 1u;
  uint32_t const slot = e.ref & kSlotMask;
  if (t.in_mesh) {
    for (uint32_t k = 0; k < cnt; k++) {
      const TriSlot& T = S.tris[slot + k];
      ts.tris++;
      float tt, b0, b1, b2;
      Ray const& lr = t.w;
      if (tri_test(T, lr, t.mr, h.z, tt, b0, b1, b2)) {
        h.z = tt;
        h.obj = t.cur;
        h.face = __float_as_uint(T.v0[3]);
        h.b0 = b0;
        h.b1 = b1;
        h.b2 = b2;
        h.pl = ray_at(lr, tt);
        h.inside = t.cur_inside;
        h.exit = t.cur_exit;
        t.hit_any = true;
        if (any) return true;
      }
    }
    return st.sp == 0;
  }
  uint32_t const i = S.tlas_objects[slot];
  if (cnt > 1) {
    if (st.sp + 1 > kSplitCap) {
      ts.flags |= 1u;
      return true;
    }
    st.push(StackEntry{kLeafBit | ((cnt - 2u) << 28) | (slot + 1u), e.t});
  }
  if (i == t.skip || i >= t.ilimit) return st.sp == 0;
  ts.insts++;
  const DevObject& ob = S.objects[i];
  bool const low = !any && h.obj != UINT32_MAX && i < h.obj;
  float const z_saved = h.z;
  if (low) h.z = prev_float(z_saved);
  Ray const li = to_local(ob, t.w);
  if (ob.type != LGPU_OBJ_TRIMESH) {
    float tt;
    f3 x;
    bool hit;
    if (ob.type == LGPU_OBJ_SPHERE) {
      hit = sphere_test(li, h.z, tt);
      if (hit) x = ray_at(li, tt);
    } else {
      hit = plane_test(li, h.z, tt, x);
    }
    if (hit) {
      h.z = tt;
      h.obj = i;
      h.face = UINT32_MAX;
      h.pl = x;
      h.inside = false;
      t.hit_any = true;
      if (any) return true;
    } else if (low) {
      h.z = z_saved;
    }
    return st.sp == 0;
  }
  const DevMesh& m = S.meshes[ob.mesh];
  bool inside;
  float ex;
  float r0 = aabb_scalar(m.bounds, li, h.z, inside, ex);
  if (r0 != kFltMax && inside) t.n_inside++;
  if (r0 != kFltMax && !any && inside) r0 = kBias;
  if (r0 == kFltMax || r0 > h.z) {
    if (low) h.z = z_saved;
    return st.sp == 0;
  }
  if (st.sp + 2 > kSplitCap) {
    ts.flags |= 1u;
    return true;
  }
  st.ws[0] = t.w.p.x;
  st.ws[128] = t.w.p.y;
  st.ws[2 * 128] = t.w.p.z;
  st.ws[3 * 128] = t.w.u.x;
  st.ws[4 * 128] = t.w.u.y;
  st.ws[5 * 128] = t.w.u.z;
  st.ws[6 * 128] = t.w.inv.x;
  st.ws[7 * 128] = t.w.inv.y;
  st.ws[8 * 128] = t.w.inv.z;
  t.w = li;
  t.mr = cross3(li.p, li.u);
  t.cur = i;
  t.cur_inside = inside;
  t.cur_exit = ex;
  t.zs = z_saved;
  t.lowered = low;
  t.in_mesh = true;
  st.push(StackEntry{kMarker, 0.f});
  st.push(StackEntry{m.trav_root, r0});
  return false;
}

// intersect::scene for the wavefront kernels: the instance BVH through
// trace_tlas, the reference's linear object loop (nested traversal, local
// stack) for reference order, tiny scenes and the order-dependent case.
template <bool ANY>
__device__ __forceinline__ bool scene_trace(const DevScene& S, const Ray& w, HitRec& h, uint32_t skip,
                                            bool reference_order, SplitStack& st, StackEntry* lstack,
                                            StackEntry* ltstack, TravStats& ts) {
  if (reference_order || S.n_objects <= 4)
    return scene_hit<ANY>(S, w, h, skip, true, lstack, ltstack, ts);
  HitRec const h0 = h;
  bool hit = trace_tlas<ANY>(S, w, h, skip, st, ts);
  if (!ANY && hit && h.inside && h.exit > h.z) {
    h = h0;
    hit = scene_hit<false>(S, w, h, skip, true, lstack, ltstack, ts);
  }
  return hit;
}

}  // namespace lgpu
