// lgpu_intersect.cuh — ray/scene intersection on the device.
//
// Every arithmetic step here is one correctly rounded IEEE single-precision
// operation (__fadd_rn/__fmul_rn/__fdiv_rn, no contraction) in the order the
// reference evaluates it, so that hit distances, hit points, normals and hit
// ids are bit-identical to intersect::scene (cg.hpp:1469-1489) on the same
// ray.  The wide-BVH traversal visits children in the reference's order
// (far-to-near stable sort, cg.hpp:1436-1437).
#pragma once

#include <float.h>
#include <stdint.h>

#include "lgpu_scene.h"

namespace lgpu {

// constants of the reference (numli.hpp, cg.hpp:1189)
constexpr float kEps = 0x1p-23f;            // ε<float>
constexpr float kBias = 0x1.6a09e6p-12f;    // constexprSqrt(ε<float>)
constexpr float kPi = 0x1.921fb6p+1f;       // π<float>
constexpr float kInvPi = 0x1.45f306p-2f;    // 1/π<float>
constexpr float kFltMax = FLT_MAX;          // UB<float>

struct f3 {
  float x, y, z;
};

__device__ __forceinline__ float ad(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sb(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float ml(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float dv(float a, float b) { return __fdiv_rn(a, b); }

__device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 add3(f3 a, f3 b) { return f3{ad(a.x, b.x), ad(a.y, b.y), ad(a.z, b.z)}; }
__device__ __forceinline__ f3 sub3(f3 a, f3 b) { return f3{sb(a.x, b.x), sb(a.y, b.y), sb(a.z, b.z)}; }
__device__ __forceinline__ f3 scl3(f3 a, float s) { return f3{ml(a.x, s), ml(a.y, s), ml(a.z, s)}; }
__device__ __forceinline__ f3 neg3(f3 a) { return f3{-a.x, -a.y, -a.z}; }
// bra.hpp:390-393 operator| : x0*y0 + x1*y1 + x2*y2, left to right
__device__ __forceinline__ float dot3(f3 a, f3 b) {
  return ad(ad(ml(a.x, b.x), ml(a.y, b.y)), ml(a.z, b.z));
}
// bra.hpp:386-388 operator^
__device__ __forceinline__ f3 cross3(f3 a, f3 b) {
  return f3{sb(ml(a.y, b.z), ml(a.z, b.y)), sb(ml(a.z, b.x), ml(a.x, b.z)),
            sb(ml(a.x, b.y), ml(a.y, b.x))};
}
// ℝn::len2 (bra.hpp:202-207): sum from 0
__device__ __forceinline__ float len2(f3 a) {
  return ad(ad(ad(0.f, ml(a.x, a.x)), ml(a.y, a.y)), ml(a.z, a.z));
}
// ℝn::normalized (bra.hpp:209-216): divide by sqrt(len2)
__device__ __forceinline__ f3 normalized(f3 a) {
  float const l = __fsqrt_rn(len2(a));
  return f3{dv(a.x, l), dv(a.y, l), dv(a.z, l)};
}

// nl::cg::ray (cg.hpp:351-371)
struct Ray {
  f3 p, u, inv;
};
__device__ __forceinline__ float inv_or_max(float u) {
  return u != 0.f ? dv(1.f, u) : kFltMax;
}
__device__ __forceinline__ Ray make_ray(f3 p, f3 u) {
  return Ray{p, u, f3{inv_or_max(u.x), inv_or_max(u.y), inv_or_max(u.z)}};
}

// ℝ4x4 * ℝ4 (bra.hpp:326-336) on rows 0-2, w = 1 (points) or 0 (vectors)
__device__ __forceinline__ float row4(const float* R, f3 v, float w) {
  float s = 0.f;
  s = ad(s, ml(R[0], v.x));
  s = ad(s, ml(R[1], v.y));
  s = ad(s, ml(R[2], v.z));
  s = ad(s, ml(R[3], w));
  return s;
}
__device__ __forceinline__ f3 xform(const float* R, f3 v, float w) {
  return f3{row4(R, v, w), row4(R + 4, v, w), row4(R + 8, v, w)};
}
// transform::normalToWorld (cg.hpp:442-443): M_inv^T (3x3) * n
__device__ __forceinline__ f3 normal_to_world(const float* Minv, f3 n) {
  f3 r;
  float s;
  s = 0.f; s = ad(s, ml(Minv[0], n.x)); s = ad(s, ml(Minv[4], n.y)); s = ad(s, ml(Minv[8], n.z)); r.x = s;
  s = 0.f; s = ad(s, ml(Minv[1], n.x)); s = ad(s, ml(Minv[5], n.y)); s = ad(s, ml(Minv[9], n.z)); r.y = s;
  s = 0.f; s = ad(s, ml(Minv[2], n.x)); s = ad(s, ml(Minv[6], n.y)); s = ad(s, ml(Minv[10], n.z)); r.z = s;
  return r;
}
// transform::toLocal (cg.hpp:436-437)
__device__ __forceinline__ Ray to_local(const DevObject& o, const Ray& w) {
  return make_ray(xform(o.M_inv, w.p, 1.f), xform(o.M_inv, w.u, 0.f));
}

// orthonormalBasisOf (cg.hpp:384-404)
struct Basis {
  f3 x, y, z;
};
__device__ __forceinline__ Basis orthonormal_basis(f3 v) {
  f3 const e2 = normalized(v);
  float const x = e2.x, y = e2.y, z = e2.z;
  Basis B;
  if (z >= y) {
    float const a = dv(1.f, ad(1.f, z));
    float const b = ml(ml(-x, y), a);
    B.x = f3{sb(1.f, ml(ml(x, x), a)), b, -x};
    B.y = f3{b, sb(1.f, ml(ml(y, y), a)), -y};
  } else {
    float const a = dv(1.f, ad(1.f, y));
    float const b = ml(ml(-x, z), a);
    B.x = f3{b, -z, sb(1.f, ml(ml(z, z), a))};
    B.y = f3{sb(1.f, ml(ml(x, x), a)), -x, b};
  }
  B.z = e2;
  return B;
}

// Closest hit found so far (intersect functions keep the world-space
// conversion for the end, from the same operands).
struct HitRec {
  float z;        // hitinfo::z
  uint32_t obj;   // UINT32_MAX: none
  uint32_t face;  // trimesh face, UINT32_MAX otherwise
  float b0, b1, b2;
  f3 pl;  // local-space hit point
  // for the instance-BVH order: the hit object's bounds contained the ray
  // origin, and the distance at which the ray leaves them
  bool inside;
  float exit;
};

// intersect::aabb (cg.hpp:1268-1286): scalar slab test for mesh bounds.
// When the origin is inside the box (tmin < BIAS) it returns the exit
// distance; `inside` and `exit_t` report that case.
__device__ __forceinline__ float aabb_scalar(const float* bb, const Ray& r, float t_max, bool& inside,
                                             float& exit_t) {
  float t0x = ml(sb(bb[0], r.p.x), r.inv.x);
  float t1x = ml(sb(bb[3], r.p.x), r.inv.x);
  float t0y = ml(sb(bb[1], r.p.y), r.inv.y);
  float t1y = ml(sb(bb[4], r.p.y), r.inv.y);
  float t0z = ml(sb(bb[2], r.p.z), r.inv.z);
  float t1z = ml(sb(bb[5], r.p.z), r.inv.z);
  if (t0x > t1x) { float s = t0x; t0x = t1x; t1x = s; }
  if (t0y > t1y) { float s = t0y; t0y = t1y; t1y = s; }
  if (t0z > t1z) { float s = t0z; t0z = t1z; t1z = s; }
  // nl::max(a,b) = a>=b?a:b, nl::min(a,b) = a<=b?a:b (numli.hpp:60-61)
  float const myz = t0y >= t0z ? t0y : t0z;
  float const tmin = t0x >= myz ? t0x : myz;
  float const nyz = t1y <= t1z ? t1y : t1z;
  float const tmax = t1x <= nyz ? t1x : nyz;
  inside = false;
  exit_t = tmax;
  if (tmax < kBias || tmax <= tmin || tmin > t_max) return kFltMax;
  inside = tmin < kBias;
  return inside ? tmax : tmin;
}

// Entry distance of the ray segment [BIAS, t_max] into a box, or FLT_MAX if
// the segment misses it (conservative culling for the instance BVH root).
__device__ __forceinline__ float segment_box_entry(const float* bb, const Ray& r, float t_max) {
  float tmin = kBias, tmax = t_max;
  float const a[3] = {r.p.x, r.p.y, r.p.z}, iv[3] = {r.inv.x, r.inv.y, r.inv.z};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    float t0 = ml(sb(bb[k], a[k]), iv[k]);
    float t1 = ml(sb(bb[3 + k], a[k]), iv[k]);
    if (t0 > t1) { float s = t0; t0 = t1; t1 = s; }
    tmin = t0 > tmin ? t0 : tmin;
    tmax = t1 < tmax ? t1 : tmax;
  }
  return tmin <= tmax ? tmin : kFltMax;
}

__device__ __forceinline__ float prev_float(float z) {
  return __int_as_float(__float_as_int(z) - 1);
}

// intersect::aabb_avx2 (cg.hpp:1295-1337) for child c of a wide node:
// _mm256_max_ps(a,b) = a>b?a:b and _mm256_min_ps(a,b) = a<b?a:b (the second
// operand wins on NaN); a miss returns 0.
__device__ __forceinline__ float child_box_t(const WideNode& nd, int c, const Ray& r,
                                             bool nx, bool ny, bool nz, float t_max, float slack = 1.f) {
  float const bminx = nx ? nd.hix[c] : nd.lox[c];
  float const bmaxx = nx ? nd.lox[c] : nd.hix[c];
  float const bminy = ny ? nd.hiy[c] : nd.loy[c];
  float const bmaxy = ny ? nd.loy[c] : nd.hiy[c];
  float const bminz = nz ? nd.hiz[c] : nd.loz[c];
  float const bmaxz = nz ? nd.loz[c] : nd.hiz[c];
  float const dminx = ml(sb(bminx, r.p.x), r.inv.x);
  float const dmaxx = ml(sb(bmaxx, r.p.x), r.inv.x);
  float const dminy = ml(sb(bminy, r.p.y), r.inv.y);
  float const dmaxy = ml(sb(bmaxy, r.p.y), r.inv.y);
  float const dminz = ml(sb(bminz, r.p.z), r.inv.z);
  float const dmaxz = ml(sb(bmaxz, r.p.z), r.inv.z);
  float tmin = kBias, tmax = t_max;
  // no slab value is NaN (inv is finite or ±FLT_MAX, b - p is finite) and a
  // ±0 never decides a hit (tmin starts at kBias > 0), so fmaxf/fminf
  // return what the reference's compare-and-select does
  tmin = fmaxf(fmaxf(fmaxf(tmin, dminx), dminy), dminz);
  tmax = fminf(fminf(fminf(tmax, dmaxx), dmaxy), dmaxz);
  return tmin <= tmax * slack ? tmin : 0.f;
}

// All 8 child boxes of a wide node at once (the results of child_box_t):
// the near and far plane rows of each axis are chosen once from the signs
// of the ray's direction and read as float4.  No slab value is NaN (inv is
// finite or ±FLT_MAX, b - p is finite) and a ±0 never decides a hit (tmin
// starts at kBias > 0), so fmaxf/fminf return what the reference's
// compare-and-select does.
__device__ __forceinline__ void node_boxes_t(const WideNode& nd, const Ray& r, float t_max, float (&t)[8],
                                             float slack = 1.f) {
  bool const nx = r.inv.x < 0.f, ny = r.inv.y < 0.f, nz = r.inv.z < 0.f;
  const float4* const nrx = reinterpret_cast<const float4*>(nx ? nd.hix : nd.lox);
  const float4* const frx = reinterpret_cast<const float4*>(nx ? nd.lox : nd.hix);
  const float4* const nry = reinterpret_cast<const float4*>(ny ? nd.hiy : nd.loy);
  const float4* const fry = reinterpret_cast<const float4*>(ny ? nd.loy : nd.hiy);
  const float4* const nrz = reinterpret_cast<const float4*>(nz ? nd.hiz : nd.loz);
  const float4* const frz = reinterpret_cast<const float4*>(nz ? nd.loz : nd.hiz);
  // four children at a time: the six float4 of a half and their tests
#pragma unroll
  for (int h = 0; h < 2; h++) {
    float4 const a = nrx[h], b = frx[h], c = nry[h], d = fry[h], e = nrz[h], f = frz[h];
    float const bnx[4] = {a.x, a.y, a.z, a.w}, bfx[4] = {b.x, b.y, b.z, b.w};
    float const bny[4] = {c.x, c.y, c.z, c.w}, bfy[4] = {d.x, d.y, d.z, d.w};
    float const bnz[4] = {e.x, e.y, e.z, e.w}, bfz[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      float const tmin =
          fmaxf(fmaxf(fmaxf(kBias, ml(sb(bnx[k], r.p.x), r.inv.x)), ml(sb(bny[k], r.p.y), r.inv.y)),
                ml(sb(bnz[k], r.p.z), r.inv.z));
      float const tmax =
          fminf(fminf(fminf(t_max, ml(sb(bfx[k], r.p.x), r.inv.x)), ml(sb(bfy[k], r.p.y), r.inv.y)),
                ml(sb(bfz[k], r.p.z), r.inv.z));
      t[4 * h + k] = tmin <= tmax * slack ? tmin : 0.f;
    }
    // keeps the second half's loads after the first half's tests (fewer
    // live registers)
    asm volatile("" ::: "memory");
  }
}

struct StackEntry {
  uint32_t ref;
  float t;
};

// Per-thread traversal counters: flags (kTravOverflow, kTravLocalStack) and
// the work done, for the roofline's algorithmic byte count.
struct TravStats {
  uint32_t flags;
  uint32_t nodes;  // wide nodes whose 8 child boxes were tested
  uint32_t tris;   // triangle tests
  uint32_t insts;  // object (instance) tests
};

// Position of each hit child in the far-to-near order: d goes before c when
// t[d] > t[c], or t[d] == t[c] and d < c.  One comparison per pair; a miss
// has t = 0, below every hit, so it does not shift a hit's rank.
__device__ __forceinline__ void child_ranks(const float (&t)[8], int (&rank)[8]) {
#pragma unroll
  for (int c = 0; c < 8; c++) rank[c] = 0;
#pragma unroll
  for (int c = 1; c < 8; c++)
#pragma unroll
    for (int d = 0; d < c; d++) {
      bool const d_first = t[d] >= t[c];
      rank[c] += d_first ? 1 : 0;
      rank[d] += d_first ? 0 : 1;
    }
}

// Tests the children of an interior node and pushes the hit ones so that
// the nearest is on top; equal distances keep child order, as the
// reference's insertion-sorted std::sort of <= 8 elements does
// (cg.hpp:1427-1437).  Returns false if the stack would overflow.
__device__ __forceinline__ bool push_children(const WideNode& nd, const Ray& r, float t_max,
                                              StackEntry* stack, int& sp, int cap) {
  bool const nx = r.inv.x < 0.f, ny = r.inv.y < 0.f, nz = r.inv.z < 0.f;
  float t[8];
  uint32_t ref[8];
#pragma unroll
  for (int c = 0; c < 8; c++) {
    ref[c] = nd.child[c];
    t[c] = (ref[c] != kEmptyChild) ? child_box_t(nd, c, r, nx, ny, nz, t_max) : 0.f;
  }
  int hits = 0;
#pragma unroll
  for (int c = 0; c < 8; c++) hits += (t[c] != 0.f) ? 1 : 0;
  if (sp + hits > cap) return false;
  int rank[8];
  child_ranks(t, rank);
#pragma unroll
  for (int c = 0; c < 8; c++)
    if (t[c] != 0.f) stack[sp + rank[c]] = StackEntry{ref[c], t[c]};
  sp += hits;
  return true;
}

// intersect::triangle (cg.hpp:1341-1379); mr = l_ray.p ^ l_ray.u.
__device__ __forceinline__ bool tri_test(const TriSlot& T, const Ray& l, f3 mr, float z,
                                         float& t_out, float& b0, float& b1, float& b2) {
  f3 const v0 = mk(T.v0[0], T.v0[1], T.v0[2]);
  f3 const v1 = mk(T.v1[0], T.v1[1], T.v1[2]);
  f3 const v2 = mk(T.v2[0], T.v2[1], T.v2[2]);
  f3 const e0 = sub3(v1, v0);
  f3 const e2 = sub3(v0, v2);
  f3 const n = cross3(e2, e0);
  float const D = dot3(l.u, n);
  if (fabsf(D) < kEps) return false;
  f3 const m0 = cross3(v0, e0);
  float const s0 = ad(dot3(l.u, m0), dot3(e0, mr));
  if (ml(s0, D) < 0.f) return false;
  f3 const e1 = sub3(v2, v1);
  f3 const m1 = cross3(v1, e1);
  float const s1 = ad(dot3(l.u, m1), dot3(e1, mr));
  if (ml(s1, D) < 0.f) return false;
  f3 const m2 = cross3(v2, e2);
  float const s2 = ad(dot3(l.u, m2), dot3(e2, mr));
  if (ml(s2, D) < 0.f) return false;
  if (fabsf(ad(ad(s0, s1), s2)) < kEps) return false;
  float const inv_D = dv(1.f, D);
  float const t = ml(dot3(sub3(v0, l.p), n), inv_D);
  if (t < kBias || z < t) return false;
  t_out = t;
  b0 = ml(s1, inv_D);
  b1 = ml(s2, inv_D);
  b2 = ml(s0, inv_D);
  return true;
}

// ray(t) = p + t*u (cg.hpp:368)
__device__ __forceinline__ f3 ray_at(const Ray& r, float t) { return add3(r.p, scl3(r.u, t)); }

// intersect::sphere (cg.hpp:1196-1241), hit test part
__device__ __forceinline__ bool sphere_test(const Ray& l, float z, float& t_out) {
  float const a = dot3(l.u, l.u);
  float const b = ml(2.f, dot3(l.p, l.u));
  float const c = sb(dot3(l.p, l.p), 1.f);
  float const D = sb(ml(b, b), ml(ml(4.f, a), c));
  if (D < ml(0.1f, kBias)) return false;
  float const inv_2a = dv(0.5f, a);
  float const sq = __fsqrt_rn(D);
  float const tp = ml(ad(-b, sq), inv_2a);
  float const tm = ml(sb(-b, sq), inv_2a);
  float t = tm;
  if (tm < kBias) t = tp;
  if (t < kBias) return false;
  if (z < t) return false;
  t_out = t;
  return true;
}

// intersect::plane (cg.hpp:1245-1265), hit test part
__device__ __forceinline__ bool plane_test(const Ray& l, float z, float& t_out, f3& x_out) {
  if (l.u.z == 0.f) return false;
  float const t = dv(-l.p.z, l.u.z);
  f3 const x = ray_at(l, t);
  if (x.x < -1.f || x.x > 1.f || x.y < -1.f || x.y > 1.f || t < kBias || t > z) return false;
  t_out = t;
  x_out = x;
  return true;
}

// Traversal orders.  kRefOrder reproduces intersect::scene's linear object
// loop; kTlasClosest / kTlasAny visit objects through the instance BVH.
enum Order { kRefOrder = 0, kTlasClosest = 1, kTlasAny = 2 };

// intersect::trimesh (cg.hpp:1382-1460) on one instance; ANY stops at the
// first accepted triangle (shadow rays only need the boolean).
//
// The reference pushes the mesh root with the value intersect::aabb returns,
// which is the box's EXIT distance when the ray starts inside the bounds;
// the root is then skipped if that exit lies beyond the closest hit so far
// (cg.hpp:1393, 1414).  Hits inside such a mesh are lost depending on which
// objects were tested before it.  kRefOrder and the shadow-ray orders keep
// that rule as is.  kTlasClosest tests such a mesh in full and records in
// the hit that it was an inside-bounds object, so that scene_hit can detect
// when the reference's object order could have changed the answer.
template <bool ANY>
__device__ __forceinline__ bool trimesh_hit(const DevScene& S, uint32_t obj_id, const DevObject& ob,
                                            const Ray& w, HitRec& h, StackEntry* stack,
                                            TravStats& ts, int order) {
  Ray const l = to_local(ob, w);
  const DevMesh& m = S.meshes[ob.mesh];
  bool inside;
  float exit_t;
  float t0 = aabb_scalar(m.bounds, l, h.z, inside, exit_t);
  if (t0 == kFltMax) return false;
  if (order == kTlasClosest && inside) t0 = kBias;
  f3 const mr = cross3(l.p, l.u);
  int sp = 0;
  stack[sp++] = StackEntry{m.root, t0};
  bool hit_any = false;
  while (sp > 0) {
    StackEntry const e = stack[--sp];
    if (e.t > h.z) continue;
    if (!(e.ref & kLeafBit)) {
      const WideNode& nd = S.nodes[e.ref];
      ts.nodes++;
      if (!push_children(nd, l, h.z, stack, sp, kStackCap)) {
        ts.flags |= 1u;
        break;
      }
      continue;
    }
    uint32_t const count = ((e.ref >> 28) & 7u) + 1u;
    uint32_t const slot = e.ref & kSlotMask;
    for (uint32_t k = 0; k < count; k++) {
      const TriSlot& T = S.tris[slot + k];
      ts.tris++;
      float t, b0, b1, b2;
      if (tri_test(T, l, mr, h.z, t, b0, b1, b2)) {
        h.z = t;
        h.obj = obj_id;
        h.face = __float_as_uint(T.v0[3]);
        h.b0 = b0;
        h.b1 = b1;
        h.b2 = b2;
        h.pl = ray_at(l, t);
        h.inside = inside;
        h.exit = exit_t;
        hit_any = true;
        if (ANY) return true;
      }
    }
  }
  return hit_any;
}

template <bool ANY>
__device__ __forceinline__ bool object_hit(const DevScene& S, uint32_t i, const Ray& w, HitRec& h,
                                           StackEntry* stack, TravStats& ts, int order) {
  const DevObject& ob = S.objects[i];
  ts.insts++;
  if (ob.type == LGPU_OBJ_TRIMESH) return trimesh_hit<ANY>(S, i, ob, w, h, stack, ts, order);
  Ray const l = to_local(ob, w);
  float t;
  if (ob.type == LGPU_OBJ_SPHERE) {
    if (!sphere_test(l, h.z, t)) return false;
    h.z = t;
    h.obj = i;
    h.face = UINT32_MAX;
    h.pl = ray_at(l, t);
    h.inside = false;
    return true;
  }
  f3 x;
  if (!plane_test(l, h.z, t, x)) return false;
  h.z = t;
  h.obj = i;
  h.face = UINT32_MAX;
  h.pl = x;
  h.inside = false;
  return true;
}

// Whether object i can be hit by the ray at any distance: object_hit with
// an unbounded distance.  Every test object_hit makes only gets stricter as
// the distance bound shrinks, so an object that fails here fails in
// object_hit whatever hits came before it.
__device__ __forceinline__ bool object_may_hit(const DevScene& S, uint32_t i, const Ray& w) {
  const DevObject& ob = S.objects[i];
  Ray const l = to_local(ob, w);
  if (ob.type == LGPU_OBJ_TRIMESH) {
    bool inside;
    float ex;
    return aabb_scalar(S.meshes[ob.mesh].bounds, l, kFltMax, inside, ex) != kFltMax;
  }
  float t;
  if (ob.type == LGPU_OBJ_SPHERE) return sphere_test(l, kFltMax, t);
  f3 x;
  return plane_test(l, kFltMax, t, x);
}

// intersect::scene (cg.hpp:1469-1489).  `skip` is an object index to ignore.
//
// With reference_order the objects are tested in index order like the
// reference.  Otherwise an instance-level BVH selects them, and the result
// is made identical to the index-order loop: on equal distances the object
// with the higher index wins (later objects overwrite ties, cg.hpp:1214,
// 1251, 1368), and when the winner is a mesh whose bounds contain the ray
// origin with an exit beyond the hit — the only case where the reference's
// answer depends on the object order — the ray is re-traced in index order.
// Shadow rays (ANY) need neither: the reference's per-object rule with the
// initial distance decides them in any order.
template <bool ANY>
__device__ __forceinline__ bool scene_hit(const DevScene& S, const Ray& w, HitRec& h, uint32_t skip,
                                          bool reference_order, StackEntry* stack,
                                          StackEntry* tstack, TravStats& ts) {
  h.inside = false;
  if (reference_order || S.n_objects <= 4) {
    bool hit_any = false;
    for (uint32_t i = 0; i < S.n_objects; i++) {
      if (i == skip) continue;
      if (object_hit<ANY>(S, i, w, h, stack, ts, kRefOrder)) {
        hit_any = true;
        if (ANY) return true;
      }
    }
    return hit_any;
  }
  int const order = ANY ? kTlasAny : kTlasClosest;
  HitRec const h0 = h;
  bool hit_any = false;
  float const t0 = segment_box_entry(S.tlas_bounds, w, h.z);
  if (t0 != kFltMax) {
    int sp = 0;
    tstack[sp++] = StackEntry{S.tlas_root, t0};
    while (sp > 0) {
      StackEntry const e = tstack[--sp];
      if (e.t > h.z) continue;
      if (!(e.ref & kLeafBit)) {
        ts.nodes++;
        if (!push_children(S.nodes[e.ref], w, h.z, tstack, sp, kTlasStackCap)) {
          ts.flags |= 1u;
          break;
        }
        continue;
      }
      uint32_t const count = ((e.ref >> 28) & 7u) + 1u;
      uint32_t const slot = e.ref & kSlotMask;
      for (uint32_t k = 0; k < count; k++) {
        uint32_t const i = S.tlas_objects[slot + k];
        if (i == skip) continue;
        if (ANY) {
          if (object_hit<true>(S, i, w, h, stack, ts, order)) return true;
          continue;
        }
        // a lower-index object loses ties: test it against the next float
        // below the current distance
        float const zs = h.z;
        bool const lowered = (h.obj != UINT32_MAX && i < h.obj);
        if (lowered) h.z = prev_float(zs);
        if (object_hit<false>(S, i, w, h, stack, ts, order)) hit_any = true;
        else if (lowered) h.z = zs;
      }
    }
  }
  if (!ANY && hit_any && h.inside && h.exit > h.z) {
    h = h0;
    hit_any = false;
    for (uint32_t i = 0; i < S.n_objects; i++) {
      if (i == skip) continue;
      if (object_hit<false>(S, i, w, h, stack, ts, kRefOrder)) hit_any = true;
    }
  }
  return hit_any;
}

// Full hit information (hitinfo) for the closest hit h of world ray w:
// the world-space conversions of intersect::sphere/plane/trimesh
// (cg.hpp:1221-1239, 1256-1263, 1449-1458).
struct HitInfo {
  float z;
  f3 p;
  Basis F;
  f3 gn;
  bool front;
  uint32_t mat, obj, face;
};

__device__ __forceinline__ HitInfo finalize_hit(const DevScene& S, const Ray& w, const HitRec& h) {
  HitInfo H;
  const DevObject& ob = S.objects[h.obj];
  H.z = h.z;
  H.obj = h.obj;
  H.face = h.face;
  H.mat = ob.mat;
  H.p = xform(ob.M, h.pl, 1.f);
  if (ob.type == LGPU_OBJ_TRIMESH) {
    const DevMesh& m = S.meshes[ob.mesh];
    const FaceShade& fs = S.shade[m.face_base + h.face];
    f3 const gnl = mk(fs.gn[0], fs.gn[1], fs.gn[2]);
    // trimeshdata::n (cg.hpp:790-794): b0*N0 + b1*N1 + b2*N2
    f3 const nz = add3(add3(scl3(mk(fs.n0[0], fs.n0[1], fs.n0[2]), h.b0),
                            scl3(mk(fs.n1[0], fs.n1[1], fs.n1[2]), h.b1)),
                       scl3(mk(fs.n2[0], fs.n2[1], fs.n2[2]), h.b2));
    f3 const ul = xform(ob.M_inv, w.u, 0.f);
    H.front = dot3(gnl, ul) < 0.f;
    H.gn = normalized(normal_to_world(ob.M_inv, gnl));
    H.F = orthonormal_basis(normal_to_world(ob.M_inv, nz));
  } else if (ob.type == LGPU_OBJ_SPHERE) {
    f3 const n = normalized(normal_to_world(ob.M_inv, h.pl));
    H.front = dot3(n, w.u) < 0.f;
    float const cos_t = n.z;
    float const sin_t = __fsqrt_rn(sb(1.f, ml(cos_t, cos_t)));
    float const phi = atan2f(n.y, n.x);
    float sin_p, cos_p;
    sincosf(phi, &sin_p, &cos_p);
    H.F.x = f3{ml(-sin_t, sin_p), ml(sin_t, cos_p), 0.f};
    H.F.y = f3{ml(cos_t, cos_p), ml(cos_t, sin_p), -sin_t};
    H.F.z = n;
    H.gn = n;
  } else {
    H.F.z = normalized(normal_to_world(ob.M_inv, mk(0.f, 0.f, 1.f)));
    H.F.x = normalized(normal_to_world(ob.M_inv, mk(0.f, 1.f, 0.f)));
    H.F.y = cross3(H.F.z, H.F.x);
    H.gn = H.F.z;
    H.front = dot3(w.u, H.F.z) < 0.f;
  }
  return H;
}

}  // namespace lgpu
