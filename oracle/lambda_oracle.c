/*
 * lambda_oracle.c — TEST INFRASTRUCTURE ONLY: a C restatement of the
 * reference's spectral path-tracing hot path.
 *
 * Each function cites the reference code it restates (file:line, relative to
 * the reference project).  It is compiled with -ffp-contract=off and without
 * FMA so that every float operation is one IEEE single-precision operation
 * in the reference's order; with the mt19937 stream the rendered image is
 * bit-identical to the reference's Renderer::render built the same way
 * (tests/test_oracle.py pins this).  With the PCG stream it draws the same
 * numbers in the same order as the device kernels, which makes it a per-path
 * oracle for them.
 *
 * The scene is an lgpu_scene (include/lambda_gpu.h); objects are tested in
 * index order and mesh BVHs are traversed in the reference's own layout.
 */
#include "lambda_oracle.h"

#include <float.h>
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "../lambda_b200/csrc/lgpu_rng.h"

#define KMAX 16
#define NBMAX 512

static const float EPS = 0x1p-23f;          /* ε<float> */
static const float BIAS = 0x1.6a09e6p-12f;  /* constexprSqrt(ε<float>), cg.hpp:1189 */
static const float PI = 0x1.921fb6p+1f;     /* π<float> */
static const float INV_PI = 0x1.45f306p-2f; /* inv_π<float> */

static int g_mt_rtl = 1;
void oracle_set_mt_arg_order(int right_to_left) { g_mt_rtl = right_to_left; }
int oracle_max_threads(void) { return omp_get_max_threads(); }

/* ---- random streams ------------------------------------------------------ */

/* std::mt19937 (Matsumoto & Nishimura 1998), seeded as
   mersenne_twister_engine::seed does with the low 32 bits of the seed. */
typedef struct {
  uint32_t mt[624];
  int idx;
} mt19937;

static void mt_seed(mt19937* g, uint64_t seed) {
  g->mt[0] = (uint32_t)seed;
  for (int i = 1; i < 624; i++)
    g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
  g->idx = 624;
}

static uint32_t mt_next(mt19937* g) {
  if (g->idx >= 624) {
    for (int i = 0; i < 624; i++) {
      uint32_t const y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
      uint32_t v = g->mt[(i + 397) % 624] ^ (y >> 1);
      if (y & 1u) v ^= 0x9908b0dfu;
      g->mt[i] = v;
    }
    g->idx = 0;
  }
  uint32_t y = g->mt[g->idx++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

typedef struct {
  int mode;
  mt19937 mt;
  uint64_t pcg;
} rng_t;

/* RNG::flt (stoch.hpp:43): uniform_real_distribution<float>(0,1) over
   generate_canonical<float,24>: float(u)/2^32, kept below 1 */
static float rng_flt(rng_t* r) {
  if (r->mode == ORACLE_RNG_PCG) return lgpu_flt(&r->pcg);
  float x = (float)mt_next(&r->mt) / 4294967296.0f;
  if (x >= 1.0f) x = nextafterf(1.0f, 0.0f);
  return x;
}
/* RNG::uint64 (stoch.hpp:42): two draws, the first one the high word */
static uint64_t rng_u64(rng_t* r) {
  if (r->mode == ORACLE_RNG_PCG) return lgpu_u64(&r->pcg);
  uint64_t const hi = mt_next(&r->mt);
  uint64_t const lo = mt_next(&r->mt);
  return (hi << 32) | lo;
}
/* two draws for f(rng.flt(), rng.flt()): returns them as (x0, x1) */
static void rng_pair(rng_t* r, float* x0, float* x1) {
  if (r->mode == ORACLE_RNG_MT19937 && g_mt_rtl) {
    *x1 = rng_flt(r);
    *x0 = rng_flt(r);
  } else {
    *x0 = rng_flt(r);
    *x1 = rng_flt(r);
  }
}

void oracle_mt_flt(uint64_t seed, uint64_t n, float* out) {
  rng_t r;
  r.mode = ORACLE_RNG_MT19937;
  mt_seed(&r.mt, seed);
  for (uint64_t i = 0; i < n; i++) out[i] = rng_flt(&r);
}
void oracle_mt_u64(uint64_t seed, uint64_t n, uint64_t* out) {
  rng_t r;
  r.mode = ORACLE_RNG_MT19937;
  mt_seed(&r.mt, seed);
  for (uint64_t i = 0; i < n; i++) out[i] = rng_u64(&r);
}

/* ---- ℝ3 (bra.hpp) ------------------------------------------------------------ */

typedef struct {
  float x, y, z;
} v3;

static v3 V3(float x, float y, float z) {
  v3 r = {x, y, z};
  return r;
}
static v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 vneg(v3 a) { return V3(-a.x, -a.y, -a.z); }
/* ℝn * T and T * ℝn: vals[i] = a[i]*s (bra.hpp:237-250) */
static v3 vmul(v3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
/* operator| (bra.hpp:390-393) */
static float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* operator^ (bra.hpp:386-388) */
static v3 vcross(v3 a, v3 b) {
  return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* len2 (bra.hpp:202-207) */
static float vlen2(v3 a) {
  float s = 0.f;
  s += a.x * a.x;
  s += a.y * a.y;
  s += a.z * a.z;
  return s;
}
/* normalized (bra.hpp:208-216) */
static v3 vnorm(v3 a) {
  float const l = sqrtf(vlen2(a));
  return V3(a.x / l, a.y / l, a.z / l);
}
static v3 vload(const float* p) { return V3(p[0], p[1], p[2]); }

/* ℝ4x4 * ℝ4 (bra.hpp:326-336), rows 0-2 */
static float row4(const float* R, v3 v, float w) {
  float s = 0.f;
  s += R[0] * v.x;
  s += R[1] * v.y;
  s += R[2] * v.z;
  s += R[3] * w;
  return s;
}
static v3 xform(const float* M, v3 v, float w) {
  return V3(row4(M, v, w), row4(M + 4, v, w), row4(M + 8, v, w));
}
/* transform::normalToWorld (cg.hpp:442-443) */
static v3 normal_to_world(const float* Mi, v3 n) {
  v3 r;
  float s;
  s = 0.f; s += Mi[0] * n.x; s += Mi[4] * n.y; s += Mi[8] * n.z; r.x = s;
  s = 0.f; s += Mi[1] * n.x; s += Mi[5] * n.y; s += Mi[9] * n.z; r.y = s;
  s = 0.f; s += Mi[2] * n.x; s += Mi[6] * n.y; s += Mi[10] * n.z; r.z = s;
  return r;
}
static v3 column(const float* M, int c) { return V3(M[c], M[4 + c], M[8 + c]); }

typedef struct {
  v3 x, y, z;
} basis;
/* basis::toBasis (cg.hpp:379) */
static v3 to_basis(const basis* B, v3 v) {
  return vadd(vadd(vmul(B->x, v.x), vmul(B->y, v.y)), vmul(B->z, v.z));
}
/* orthonormalBasisOf (cg.hpp:384-404) */
static basis orthonormal_basis(v3 v) {
  v3 const e2 = vnorm(v);
  float const x = e2.x, y = e2.y, z = e2.z;
  basis B;
  if (z >= y) {
    float const a = 1.f / (1.f + z);
    float const b = -x * y * a;
    B.x = V3(1 - x * x * a, b, -x);
    B.y = V3(b, 1 - y * y * a, -y);
  } else {
    float const a = 1.f / (1.f + y);
    float const b = -x * z * a;
    B.x = V3(b, -z, 1 - z * z * a);
    B.y = V3(1 - x * x * a, -x, b);
  }
  B.z = e2;
  return B;
}
/* bra::reflect (bra.hpp:396-397) */
static v3 reflect(v3 x, v3 a) { return vadd(vneg(x), vmul(a, 2 * vdot(x, a))); }

static float nmax(float a, float b) { return a >= b ? a : b; }
static float nmin(float a, float b) { return a <= b ? a : b; }

/* ---- ray ----------------------------------------------------------------------- */

typedef struct {
  v3 p, u, inv;
} ray;

/* ray::ray (cg.hpp:357-361) */
static ray mkray(v3 p, v3 u) {
  ray r;
  r.p = p;
  r.u = u;
  r.inv.x = u.x != 0.f ? 1.f / u.x : FLT_MAX;
  r.inv.y = u.y != 0.f ? 1.f / u.y : FLT_MAX;
  r.inv.z = u.z != 0.f ? 1.f / u.z : FLT_MAX;
  return r;
}
static v3 ray_at(const ray* r, float t) { return vadd(r->p, vmul(r->u, t)); }
/* transform::toLocal (cg.hpp:436-437) */
static ray to_local(const lgpu_transform* T, const ray* w) {
  return mkray(xform(T->M_inv, w->p, 1.f), xform(T->M_inv, w->u, 0.f));
}

/* ---- hitinfo --------------------------------------------------------------------- */

typedef struct {
  float z;
  v3 p;
  basis F;
  v3 gn;
  int front;
  uint32_t mat, obj, face;
} hitinfo;

static void hinfo_init(hitinfo* h) {
  memset(h, 0, sizeof(*h));
  h->z = FLT_MAX;
  h->obj = UINT32_MAX;
  h->face = UINT32_MAX;
}
/* hitinfo::n (cg.hpp:1147) */
static v3 hinfo_n(const hitinfo* h) { return h->front ? h->F.z : vneg(h->F.z); }

/* ---- intersection (cg.hpp:1186-1489) ---------------------------------------------- */

/* intersect::sphere (cg.hpp:1196-1241) */
static int isect_sphere(const lgpu_transform* T, uint32_t mat, uint32_t obj, const ray* w,
                        hitinfo* h) {
  ray const l = to_local(T, w);
  float const a = vdot(l.u, l.u);
  float const b = 2 * vdot(l.p, l.u);
  float const c = vdot(l.p, l.p) - 1.f;
  float const D = b * b - 4 * a * c;
  if (D < .1f * BIAS) return 0;
  float const inv_2a = .5f / a;
  float const tp = (-b + sqrtf(D)) * inv_2a;
  float const tm = (-b - sqrtf(D)) * inv_2a;
  float t = tm;
  if (tm < BIAS) t = tp;
  if (t < BIAS) return 0;
  if (h->z < t) return 0;
  v3 const p = ray_at(&l, t);
  v3 const n = vnorm(normal_to_world(T->M_inv, p));
  int const front = vdot(n, w->u) < 0.f;
  float const ct = n.z;
  float const st = sqrtf(1.f - ct * ct);
  float const phi = atan2f(n.y, n.x);
  float const cp = cosf(phi);
  float const sp = sinf(phi);
  h->z = t;
  h->p = xform(T->M, p, 1.f);
  h->F.x = V3(-st * sp, st * cp, 0.f);
  h->F.y = V3(ct * cp, ct * sp, -st);
  h->F.z = n;
  h->gn = n;
  h->front = front;
  h->mat = mat;
  h->obj = obj;
  h->face = UINT32_MAX;
  return 1;
}

/* intersect::plane (cg.hpp:1245-1265) */
static int isect_plane(const lgpu_transform* T, uint32_t mat, uint32_t obj, const ray* w,
                       hitinfo* h) {
  ray const l = to_local(T, w);
  if (l.u.z == 0.f) return 0;
  float const t = -l.p.z / l.u.z;
  v3 const x = ray_at(&l, t);
  if (x.x < -1.f || x.x > 1.f || x.y < -1.f || x.y > 1.f || t < BIAS || t > h->z) return 0;
  h->z = t;
  h->p = xform(T->M, x, 1.f);
  h->F.z = vnorm(normal_to_world(T->M_inv, V3(0.f, 0.f, 1.f)));
  h->F.x = vnorm(normal_to_world(T->M_inv, V3(0.f, 1.f, 0.f)));
  h->F.y = vcross(h->F.z, h->F.x);
  h->gn = h->F.z;
  h->front = vdot(w->u, h->F.z) < 0.f;
  h->mat = mat;
  h->obj = obj;
  h->face = UINT32_MAX;
  return 1;
}

/* intersect::aabb (cg.hpp:1268-1286) */
static float isect_aabb(const float* bb, const ray* r, float t_max) {
  float t0x = (bb[0] - r->p.x) * r->inv.x;
  float t1x = (bb[3] - r->p.x) * r->inv.x;
  float t0y = (bb[1] - r->p.y) * r->inv.y;
  float t1y = (bb[4] - r->p.y) * r->inv.y;
  float t0z = (bb[2] - r->p.z) * r->inv.z;
  float t1z = (bb[5] - r->p.z) * r->inv.z;
  float s;
  if (t0x > t1x) { s = t0x; t0x = t1x; t1x = s; }
  if (t0y > t1y) { s = t0y; t0y = t1y; t1y = s; }
  if (t0z > t1z) { s = t0z; t0z = t1z; t1z = s; }
  float const tmin = nmax(t0x, nmax(t0y, t0z));
  float const tmax = nmin(t1x, nmin(t1y, t1z));
  if (tmax < BIAS || tmax <= tmin || tmin > t_max) return FLT_MAX;
  return tmin < BIAS ? tmax : tmin;
}

/* intersect::aabb_avx2 (cg.hpp:1295-1337): _mm256_max_ps(a,b) = a>b?a:b,
   _mm256_min_ps(a,b) = a<b?a:b, miss = 0 */
static void isect_aabb8(const float* bbs, const ray* r, float t_max, float* t) {
  int const mx = r->inv.x < 0.f, my = r->inv.y < 0.f, mz = r->inv.z < 0.f;
  for (int c = 0; c < 8; c++) {
    float const ix = bbs[0 * 8 + c], iy = bbs[1 * 8 + c], iz = bbs[2 * 8 + c];
    float const sx = bbs[3 * 8 + c], sy = bbs[4 * 8 + c], sz = bbs[5 * 8 + c];
    float const bminx = mx ? sx : ix, bmaxx = mx ? ix : sx;
    float const bminy = my ? sy : iy, bmaxy = my ? iy : sy;
    float const bminz = mz ? sz : iz, bmaxz = mz ? iz : sz;
    float const dminx = (bminx - r->p.x) * r->inv.x, dmaxx = (bmaxx - r->p.x) * r->inv.x;
    float const dminy = (bminy - r->p.y) * r->inv.y, dmaxy = (bmaxy - r->p.y) * r->inv.y;
    float const dminz = (bminz - r->p.z) * r->inv.z, dmaxz = (bmaxz - r->p.z) * r->inv.z;
    float tmin = BIAS, tmax = t_max;
    tmin = dminx > tmin ? dminx : tmin;
    tmax = dmaxx < tmax ? dmaxx : tmax;
    tmin = dminy > tmin ? dminy : tmin;
    tmax = dmaxy < tmax ? dmaxy : tmax;
    tmin = dminz > tmin ? dminz : tmin;
    tmax = dmaxz < tmax ? dmaxz : tmax;
    t[c] = tmin <= tmax ? tmin : 0.f;
  }
}

static v3 mesh_v(const lgpu_mesh* m, uint32_t face, int k) {
  return vload(m->V + 3 * (size_t)m->F[(size_t)face * m->f_stride + k]);
}
static v3 mesh_n(const lgpu_mesh* m, uint32_t face, int k) {
  return vload(m->N + 3 * (size_t)m->F[(size_t)face * m->f_stride + 3 + k]);
}

/* intersect::triangle (cg.hpp:1341-1379); hinfo p/gn/F.z in local space */
static int isect_triangle(uint32_t face, const lgpu_mesh* m, const ray* l, hitinfo* h) {
  v3 const v0 = mesh_v(m, face, 0), v1 = mesh_v(m, face, 1), v2 = mesh_v(m, face, 2);
  v3 const e0 = vsub(v1, v0);
  v3 const e2 = vsub(v0, v2);
  v3 const n = vcross(e2, e0);
  float const D = vdot(l->u, n);
  if (fabsf(D) < EPS) return 0;
  v3 const mr = vcross(l->p, l->u);
  v3 const m0 = vcross(v0, e0);
  float const s0 = vdot(l->u, m0) + vdot(e0, mr);
  if (s0 * D < 0.f) return 0;
  v3 const e1 = vsub(v2, v1);
  v3 const m1 = vcross(v1, e1);
  float const s1 = vdot(l->u, m1) + vdot(e1, mr);
  if (s1 * D < 0.f) return 0;
  v3 const m2 = vcross(v2, e2);
  float const s2 = vdot(l->u, m2) + vdot(e2, mr);
  if (s2 * D < 0.f) return 0;
  if (fabsf(s0 + s1 + s2) < EPS) return 0;
  float const inv_D = 1.f / D;
  float const t = vdot(vsub(v0, l->p), n) * inv_D;
  if (t < BIAS || h->z < t) return 0;
  float const b0 = s1 * inv_D, b1 = s2 * inv_D, b2 = s0 * inv_D;
  h->z = t;
  h->p = ray_at(l, t);
  h->gn = vload(m->GN + 3 * (size_t)face);
  /* trimeshdata::n (cg.hpp:790-794) */
  h->F.z = vadd(vadd(vmul(mesh_n(m, face, 0), b0), vmul(mesh_n(m, face, 1), b1)),
                vmul(mesh_n(m, face, 2), b2));
  h->front = vdot(h->gn, l->u) < 0.f;
  h->face = face;
  return 1;
}

typedef struct {
  uint32_t node;
  float t;
} sentry;

/* intersect::trimesh (cg.hpp:1382-1460) */
static int isect_trimesh(const lgpu_scene* sc, const lgpu_object* ob, uint32_t obj, const ray* w,
                         hitinfo* h) {
  const lgpu_mesh* m = &sc->meshes[ob->mesh];
  ray const l = to_local(&ob->T, w);
  float const t0 = isect_aabb(m->bounds, &l, h->z);
  if (t0 == FLT_MAX) return 0;
  int hit_any = 0;
  sentry stack[64 + 8];
  int sp = 0;
  stack[sp].node = 0;
  stack[sp].t = t0;
  sp++;
  while (sp > 0) {
    sentry const e = stack[--sp];
    if (e.t > h->z) continue;
    uint32_t const data = m->nodes[2 * (size_t)e.node + 1];
    uint32_t const idx = (data & 0xfffffff0u) >> 4;
    uint32_t const cnt = ((data & 0xeu) >> 1) + 1;
    if (!(data & 1u)) {
      float tc[8];
      isect_aabb8(m->bbs + 48 * (size_t)m->nodes[2 * (size_t)e.node], &l, h->z, tc);
      sentry vals[8];
      int hits = 0;
      for (uint32_t i = 0; i < cnt; i++)
        if (tc[i] != 0.f) {
          vals[hits].node = idx + i;
          vals[hits].t = tc[i];
          hits++;
        }
      /* std::sort far-to-near: an insertion sort for <= 8 elements, stable */
      for (int i = 1; i < hits; i++) {
        sentry const v = vals[i];
        int j = i;
        while (j > 0 && v.t > vals[j - 1].t) {
          vals[j] = vals[j - 1];
          j--;
        }
        vals[j] = v;
      }
      if (sp + hits > 64) abort(); /* the reference's stack[64] would overflow */
      for (int i = 0; i < hits; i++) stack[sp++] = vals[i];
      continue;
    }
    for (uint32_t i = 0; i < cnt; i++) hit_any |= isect_triangle(m->prim_idxs[idx + i], m, &l, h);
  }
  if (!hit_any) return 0;
  h->p = xform(ob->T.M, h->p, 1.f);
  h->gn = vnorm(normal_to_world(ob->T.M_inv, h->gn));
  h->F = orthonormal_basis(normal_to_world(ob->T.M_inv, h->F.z));
  h->mat = ob->mat;
  h->obj = obj;
  return 1;
}

/* intersect::scene (cg.hpp:1469-1489) */
static int isect_scene(const lgpu_scene* sc, const ray* r, hitinfo* h, uint32_t skip) {
  int hit_any = 0;
  for (uint32_t i = 0; i < sc->n_objects; i++) {
    if (i == skip) continue;
    const lgpu_object* ob = &sc->objects[i];
    int hit = 0;
    if (ob->type == LGPU_OBJ_SPHERE) hit = isect_sphere(&ob->T, ob->mat, i, r, h);
    else if (ob->type == LGPU_OBJ_PLANE) hit = isect_plane(&ob->T, ob->mat, i, r, h);
    else hit = isect_trimesh(sc, ob, i, r, h);
    hit_any |= hit;
  }
  return hit_any;
}

void oracle_intersect(const lgpu_scene* sc, const float* rays, uint64_t n, lgpu_hit* out) {
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < (int64_t)n; i++) {
    const float* q = rays + 6 * i;
    ray const r = mkray(vload(q), vload(q + 3));
    hitinfo h;
    hinfo_init(&h);
    lgpu_hit* o = &out[i];
    memset(o, 0, sizeof(*o));
    if (isect_scene(sc, &r, &h, UINT32_MAX)) {
      o->t = h.z;
      o->obj = h.obj;
      o->face = h.face;
      o->mat = h.mat;
      o->p[0] = h.p.x; o->p[1] = h.p.y; o->p[2] = h.p.z;
      o->n[0] = h.F.z.x; o->n[1] = h.F.z.y; o->n[2] = h.F.z.z;
      o->gn[0] = h.gn.x; o->gn[1] = h.gn.y; o->gn[2] = h.gn.z;
      o->front = (uint32_t)h.front;
    } else {
      o->t = h.z;
      o->obj = o->face = o->mat = UINT32_MAX;
    }
  }
}

/* ---- spectra (cg.hpp:241-327) ---------------------------------------------------- */

typedef struct {
  const lgpu_scene* sc;
  int K;
  uint32_t nb;
  float inf, sup, delta;
} ctx_t;

typedef struct {
  float v[KMAX];
} hero;

static const float* spectrum(const ctx_t* c, int32_t s) { return c->sc->spectra + (size_t)s * c->nb; }

/* coefficientλ::operator()(float) (cg.hpp:289-297) */
static float spec_at(const ctx_t* c, const float* v, float l) {
  if (l <= c->inf) return v[0];
  if (l >= c->sup) return v[c->nb - 1];
  float const x = (l - c->inf) / c->delta;
  uint32_t i = (uint32_t)x;
  if (i > c->nb - 2) i = c->nb - 2;
  float const t = x - (float)i;
  return (1.f - t) * v[i] + t * v[i + 1];
}
/* coefficientλ::operator()(heroλ) (cg.hpp:298-303) */
static hero spec_hero(const ctx_t* c, int32_t s, const hero* l) {
  hero r;
  const float* v = spectrum(c, s);
  for (int k = 0; k < c->K; k++) r.v[k] = spec_at(c, v, l->v[k]);
  return r;
}
static hero hscale(hero a, float s, int K) {
  for (int k = 0; k < K; k++) a.v[k] = a.v[k] * s;
  return a;
}
static hero hdivs(hero a, float s, int K) {
  for (int k = 0; k < K; k++) a.v[k] = a.v[k] / s;
  return a;
}
static hero hzero(void) {
  hero r;
  memset(&r, 0, sizeof(r));
  return r;
}

/* ---- materials (cg.hpp:921-1102) ---------------------------------------------------- */

/* blinn::F0 and fresnel on heroλ (cg.hpp:941-947) */
static hero blinn_F(const hero* eta, float cos_i, int K) {
  hero F;
  float const p5 = powf(1.f - cos_i, 5);
  for (int k = 0; k < K; k++) {
    float const n = eta->v[k];
    float const nn = n * n;
    float const f0 = ((nn - 2.f * n) + 1.f) / ((nn + 2.f * n) + 1.f);
    F.v[k] = f0 + (-f0 + 1.f) * p5;
  }
  return F;
}
static float blinn_F1(float n, float cos_i) {
  float const f0 = (n * n - 2.f * n + 1.f) / (n * n + 2.f * n + 1.f);
  return f0 + (1.f - f0) * powf(1.f - cos_i, 5);
}
/* blinn::fresnelSplit (cg.hpp:951-960) */
static void fresnel_split(const lgpu_material* m, float F, float* p_r, float* p_t) {
  float pr = m->w_r + F * m->w_t;
  float pt = (1.f - F) * m->w_t;
  float const tot = pr + pt;
  if (tot == 0.f) {
    *p_r = 1.f;
    *p_t = 0.f;
    return;
  }
  *p_r = pr / tot;
  *p_t = pt / tot;
}
static float blinnh_prob(const lgpu_material* m, float cos_h) {
  return powf(fabsf(cos_h), m->alpha + 1) * (m->alpha + 1) * .5f * INV_PI;
}
/* the half vector of i and o, or the fallback (cg.hpp:951-954) */
static v3 half_vec(v3 i, v3 o, v3 n) {
  v3 h = vadd(i, o);
  float const l2 = vlen2(h);
  if (l2 < EPS) return vnorm(vsub(n, vmul(o, vdot(n, o))));
  return V3(h.x / sqrtf(l2), h.y / sqrtf(l2), h.z / sqrtf(l2));
}
/* blinn::fdcosθ, frcosθ, ftcosθ (cg.hpp:961-966) */
static hero blinn_fd(const ctx_t* c, const lgpu_material* m, const hero* l, float cos_i) {
  return hscale(hscale(spec_hero(c, m->spectrum[0], l), INV_PI, c->K), nmax(0.f, cos_i), c->K);
}
static hero blinn_fr(const ctx_t* c, const lgpu_material* m, const hero* l, float cos_h, const hero* F) {
  hero ks = spec_hero(c, m->spectrum[1], l), kt = spec_hero(c, m->spectrum[2], l), r;
  float const pw = powf(cos_h, m->alpha);
  for (int k = 0; k < c->K; k++)
    r.v[k] = (((ks.v[k] + F->v[k] * kt.v[k]) * (m->alpha + 2)) * .125f) * INV_PI * pw;
  return r;
}
static hero blinn_ft(const ctx_t* c, const lgpu_material* m, const hero* l, float cos_h, const hero* F) {
  hero kt = spec_hero(c, m->spectrum[2], l), r;
  float const pw = powf(cos_h, m->alpha);
  for (int k = 0; k < c->K; k++)
    r.v[k] = (((kt.v[k] * (-F->v[k] + 1.f)) * (m->alpha + 2)) * .125f) * INV_PI * pw;
  return r;
}

/* thinfilm::BRDFcosθ (cg.hpp:1032-1051) */
static hero thinfilm_brdf(const ctx_t* c, const lgpu_material* m, const hero* l, v3 i, v3 o, v3 n,
                          int front) {
  if (!front || vdot(i, n) < 0.f || vdot(o, n) < 0.f) return hzero();
  v3 const h = half_vec(i, o, n);
  float const cos_i = vdot(i, h);
  hero const n1 = spec_hero(c, m->spectrum[0], l);
  hero const n2 = spec_hero(c, m->spectrum[1], l);
  float const p5 = powf(1.f - cos_i, 5);
  float const s = (m->alpha + 2) * .125f * INV_PI;
  float const pw = powf(vdot(h, n), m->alpha);
  hero r;
  for (int k = 0; k < c->K; k++) {
    float const n01 = 1.f / n1.v[k];
    float const cos_l = sqrtf(1.f - n01 * n01) * (1.f - cos_i * cos_i);
    float const cos_d = cosf(4 * PI * n1.v[k] * m->d * cos_l / l->v[k]);
    float const a01 = 1.f - n1.v[k], b01 = 1.f + n1.v[k];
    float const R0_01 = a01 * a01 / (b01 * b01);
    float const a12 = n1.v[k] - n2.v[k], b12 = n1.v[k] + n2.v[k];
    float const R0_12 = a12 * a12 / (b12 * b12);
    float const R01 = R0_01 + (-R0_01 + 1.f) * p5;
    float const R12 = R0_12 + (-R0_12 + 1.f) * p5;
    float const Ravg = 2 * sqrtf(R01 * R12);
    float const Rt = ((R01 + R12) + Ravg * cos_d) / ((R01 * R12 + 1.f) + Ravg * cos_d);
    r.v[k] = Rt * s * pw;
  }
  return r;
}

/* BxDFcosθ (cg.hpp:1088-1102) */
static hero bxdf(const ctx_t* c, const lgpu_material* m, const hero* l, v3 i, v3 o, v3 n, int front) {
  int const K = c->K;
  if (m->type == LGPU_MAT_LAMBERTIAN)
    return hscale(hscale(spec_hero(c, m->spectrum[0], l), INV_PI, K), nmax(0.f, vdot(i, n)), K);
  if (m->type == LGPU_MAT_BLINN) {
    hero eta = spec_hero(c, m->spectrum[4], l);
    if (front)
      for (int k = 0; k < K; k++) eta.v[k] = 1.f / eta.v[k];
    float const cos_i = vdot(i, n), cos_o = vdot(o, n);
    hero const F = blinn_F(&eta, cos_o, K);
    if (cos_i * cos_o > 0.f) {
      v3 const h = half_vec(i, o, n);
      hero const fd = blinn_fd(c, m, l, cos_i);
      hero const fr = blinn_fr(c, m, l, vdot(h, n), &F);
      hero r;
      for (int k = 0; k < K; k++) r.v[k] = fd.v[k] + fr.v[k];
      return r;
    }
    v3 const ht = vneg(vnorm(vadd(i, vmul(o, eta.v[0]))));
    return blinn_ft(c, m, l, fabsf(vdot(ht, n)), &F);
  }
  if (m->type == LGPU_MAT_THINFILM) return thinfilm_brdf(c, m, l, i, o, n, front);
  return hzero();
}

/* ---- sampling (cg.hpp:1497-1988) --------------------------------------------------------- */

typedef struct {
  float prob;
  v3 val;
  hero mult;
} sinfo;

/* stoch::CosHemi / UnifHemi (stoch.hpp:53-68) */
static v3 cos_hemi(float x0, float x1) {
  float const cc = 1.f - x0;
  float const ct = sqrtf(cc);
  float const st = sqrtf(1.f - cc);
  float const phi = 2.f * PI * x1;
  return V3(st * cosf(phi), st * sinf(phi), ct);
}
static v3 unif_hemi(float x0, float x1) {
  float const ct = 1.f - x0;
  float const st = sqrtf(1.f - ct * ct);
  float const phi = 2.f * PI * x1;
  return V3(st * cosf(phi), st * sinf(phi), ct);
}
/* sample::blinnh (cg.hpp:1790-1796) */
static v3 blinnh(float alpha, float x0, float x1) {
  float const ct = powf(1.f - x0, 1.f / (alpha + 1.f));
  float const st = sqrtf(1.f - ct * ct);
  float const phi = 2.f * PI * x1;
  return V3(st * cosf(phi), st * sinf(phi), ct);
}

static int occluded(const lgpu_scene* sc, v3 p, v3 d, float tmax, uint32_t skip) {
  hitinfo t;
  hinfo_init(&t);
  t.z = tmax;
  ray const r = mkray(p, d);
  return isect_scene(sc, &r, &t, skip);
}

/* sample::light (cg.hpp:1560-1732) */
static void sample_light(const ctx_t* c, const lgpu_light* L, const hero* l, const hitinfo* h,
                         rng_t* rng, sinfo* si) {
  const lgpu_scene* sc = c->sc;
  int const K = c->K;
  hero const rad = spec_hero(c, L->spectrum, l);
  if (L->type == LGPU_LIGHT_SPHERE) { /* cg.hpp:1671-1699 */
    v3 const Lv = vsub(column(L->T.M, 3), h->p);
    float const dist2 = vdot(Lv, Lv);
    float const r2 = L->size * L->size;
    float const sr = 1.f - sqrtf(nmax(0.f, 1.f - r2 / dist2));
    si->prob = 0.5f / (PI * sr);
    basis const B = orthonormal_basis(Lv);
    float const ct = nmax(0.f, 1.f - rng_flt(rng) * sr);
    float const st = sqrtf(1.f - ct * ct);
    float const phi = 2 * PI * rng_flt(rng);
    v3 const w = vadd(vadd(vmul(vmul(B.x, st), cosf(phi)), vmul(vmul(B.y, st), sinf(phi))), vmul(B.z, ct));
    si->val = w;
    float const shadow = occluded(sc, h->p, w, sqrtf(dist2), L->obj) ? 0.f : 1.f;
    si->mult = hscale(rad, shadow, K);
  } else if (L->type == LGPU_LIGHT_QUADDIR) { /* cg.hpp:1625-1655 */
    float const sx = 2.f * rng_flt(rng) - 1.f;
    float const sy = 2.f * rng_flt(rng) - 1.f;
    v3 const x = vadd(vadd(column(L->T.M, 3), vmul(column(L->T.M, 0), sx)), vmul(column(L->T.M, 1), sy));
    v3 const r = vsub(x, h->p);
    v3 const w = vnorm(r);
    si->val = w;
    float const dist2 = vdot(r, r);
    float const cs = powf(vdot(vneg(w), vnorm(column(L->T.M, 2))), L->spec);
    si->prob = nmax(1e-6f, (L->spec + 1) * .5f * INV_PI * cs * L->inv_area);
    float const shadow = occluded(sc, h->p, w, sqrtf(dist2), L->obj) ? 0.f : 1.f;
    si->mult = hscale(hscale(rad, cs, K), shadow, K);
  } else if (L->type == LGPU_LIGHT_POINT) { /* cg.hpp:1580-1601 */
    v3 const Lv = vsub(vload(L->pos), h->p);
    v3 const w = vnorm(Lv);
    si->val = w;
    si->prob = 1.f;
    float const dist = sqrtf(vlen2(Lv));
    float const shadow = occluded(sc, h->p, w, dist, UINT32_MAX) ? 0.f : 1.f;
    si->mult = hdivs(hscale(rad, shadow, K), dist * dist, K);
  } else if (L->type == LGPU_LIGHT_DIR) { /* cg.hpp:1604-1621 */
    v3 const w = vneg(vload(L->dir));
    si->val = w;
    si->prob = 1.f;
    float const shadow = occluded(sc, h->p, w, FLT_MAX, UINT32_MAX) ? 0.f : 1.f;
    si->mult = hscale(rad, shadow, K);
  } else { /* ambient, cg.hpp:1560-1577 */
    float x0, x1;
    rng_pair(rng, &x0, &x1);
    v3 d = unif_hemi(x0, x1);
    if (!h->front) d.z *= -1.f;
    si->val = to_basis(&h->F, d);
    si->prob = .5f * INV_PI;
    si->mult = rad;
  }
}

/* sample::probForLight (cg.hpp:1735-1747) */
static float prob_for_light(const ctx_t* c, const lgpu_light* L, const ray* r) {
  (void)c;
  if (L->type == LGPU_LIGHT_SPHERE) {
    hitinfo h;
    hinfo_init(&h);
    if (!isect_sphere(&L->T, 0, 0, r, &h) || !h.front) return 0.f;
    v3 const Lv = vsub(column(L->T.M, 3), r->p);
    float const dist2 = vdot(Lv, Lv);
    float const sr = (1.f - sqrtf(nmax(0.f, 1.f - L->size * L->size / dist2)));
    return .5f / (PI * sr);
  }
  if (L->type == LGPU_LIGHT_QUADDIR) {
    hitinfo h;
    hinfo_init(&h);
    int const hit = isect_plane(&L->T, 0, 0, r, &h);
    if (!hit || (hit && !h.front)) return 0.f;
    float const ct = vdot(vneg(vnorm(r->u)), h.F.z);
    return nmax(1e-6f, (L->spec + 1) * .5f * INV_PI * powf(ct, L->spec) * L->inv_area);
  }
  if (L->type == LGPU_LIGHT_AMBIENT) return .5f * INV_PI;
  return 0.f;
}

/* sample::materiali (cg.hpp:1755-1968) */
static int sample_material(const ctx_t* c, const lgpu_material* m, const hero* l, const hitinfo* h,
                           v3 o, rng_t* rng, float p, sinfo* si) {
  int const K = c->K;
  if (m->type == LGPU_MAT_LAMBERTIAN) { /* cg.hpp:1755-1777 */
    float const xi = rng_flt(rng);
    if (xi > p) return 0;
    float x0, x1;
    rng_pair(rng, &x0, &x1);
    v3 d = cos_hemi(x0, x1);
    if (!h->front) d.z *= -1.f;
    v3 const i = to_basis(&h->F, d);
    si->prob = p * fabsf(d.z) * INV_PI;
    si->val = i;
    si->mult = hscale(hscale(spec_hero(c, m->spectrum[0], l), INV_PI, K), nmax(0.f, vdot(i, hinfo_n(h))), K);
    return 1;
  }
  if (m->type == LGPU_MAT_BLINN) { /* cg.hpp:1799-1862 */
    float const lobe = rng_flt(rng);
    if (lobe >= p) return 0;
    float const pp_d = p * m->p_d, pp_spec = p * m->p_spec;
    if (lobe < pp_spec) {
      hero eta = spec_hero(c, m->spectrum[4], l);
      if (h->front)
        for (int k = 0; k < K; k++) eta.v[k] = 1.f / eta.v[k];
      float x0, x1;
      rng_pair(rng, &x0, &x1);
      v3 w = blinnh(m->alpha, x0, x1);
      if (!h->front) w.z *= -1.f;
      v3 const hv = to_basis(&h->F, w);
      v3 const iR = reflect(o, hv);
      /* transmit (cg.hpp:500-513) */
      float const ci = vdot(o, hv);
      v3 iT[KMAX];
      for (int k = 0; k < K; k++) {
        float const ct2 = -((eta.v[k] * eta.v[k]) * (1.f - ci * ci)) + 1.f;
        if (ct2 < 0.f) iT[k] = V3(0.f, 0.f, 0.f);
        else iT[k] = vsub(vmul(o, -eta.v[k]), vmul(hv, sqrtf(ct2) - eta.v[k] * ci));
      }
      hero F = blinn_F(&eta, ci, K);
      for (int k = 0; k < K; k++)
        if (iT[k].x == 0.f && iT[k].y == 0.f && iT[k].z == 0.f) F.v[k] = 1.f;
      float p_r, p_t;
      fresnel_split(m, F.v[0], &p_r, &p_t);
      if (lobe < pp_spec * p_r) {
        si->prob = pp_spec * p_r * blinnh_prob(m, w.z) * .25f;
        si->val = iR;
        si->mult = blinn_fr(c, m, l, w.z, &F);
      } else {
        si->prob = pp_spec * p_t * blinnh_prob(m, w.z) * .25f;
        si->val = iT[0];
        si->mult = blinn_ft(c, m, l, w.z, &F);
      }
      return 1;
    } else if (lobe < pp_spec + pp_d) {
      float x0, x1;
      rng_pair(rng, &x0, &x1);
      v3 d = cos_hemi(x0, x1);
      if (!h->front) d.z *= -1.f;
      v3 const i = to_basis(&h->F, d);
      si->prob = pp_d * (fabsf(d.z) * INV_PI);
      si->val = i;
      si->mult = blinn_fd(c, m, l, d.z);
      return 1;
    }
    return 0;
  }
  if (m->type == LGPU_MAT_THINFILM) { /* cg.hpp:1905-1929 */
    v3 const n = h->F.z;
    if (!h->front || vdot(o, n) < 0.f) return 0;
    float const lobe = rng_flt(rng);
    if (lobe >= p) return 0;
    float x0, x1;
    rng_pair(rng, &x0, &x1);
    v3 const w = blinnh(m->alpha, x0, x1);
    v3 const hv = to_basis(&h->F, w);
    v3 const i = reflect(o, hv);
    si->prob = p * powf(vdot(n, hv), m->alpha + 1) * (m->alpha + 1) * .5f * INV_PI * .25f;
    si->val = i;
    si->mult = thinfilm_brdf(c, m, l, i, o, n, h->front);
    return 1;
  }
  return 0;
}

/* sample::probForMateriali (cg.hpp:1971-1985) called as
   probForMateriali(λ[0], mat, hinfo, ωL, o, p) (src/renderer.cpp:136-137) */
static float prob_for_material(const ctx_t* c, const lgpu_material* m, float l0, const hitinfo* h,
                               v3 i, v3 o, float p) {
  if (m->type == LGPU_MAT_LAMBERTIAN) { /* cg.hpp:1780-1787 */
    v3 const n = hinfo_n(h);
    float const ci = vdot(i, n);
    if (vdot(i, n) < 0.f || vdot(o, n) < 0.f) return 0.f;
    return p * ci * INV_PI;
  }
  if (m->type == LGPU_MAT_BLINN) { /* probForBlinn(l, b, hinfo, o:=i, i:=o, p), cg.hpp:1865-1902 */
    v3 const bo = i, bi = o;
    v3 const n = hinfo_n(h);
    float const iv = spec_at(c, spectrum(c, m->spectrum[4]), l0);
    float const ior = h->front ? 1.f / iv : iv;
    float const cos_in = vdot(bi, n), cos_on = vdot(bo, n);
    v3 hv;
    if (cos_in * cos_on > 0.f) hv = half_vec(bi, bo, n);
    else hv = vneg(vnorm(vadd(bi, vmul(bo, ior))));
    float const cos_o = fabsf(vdot(bo, hv));
    float const F = blinn_F1(ior, cos_o);
    float p_r, p_t;
    fresnel_split(m, F, &p_r, &p_t);
    if (cos_in * cos_on > 0.f)
      return p * (m->p_d * (fabsf(cos_in) * INV_PI) + m->p_spec * p_r * blinnh_prob(m, vdot(hv, n)) * .25f);
    float const c2 = 1.f - ior * ior * (1.f - cos_o * cos_o);
    if (c2 < 0.f) return 0.f;
    return p * m->p_spec * p_t * blinnh_prob(m, vdot(hv, n)) * .25f;
  }
  if (m->type == LGPU_MAT_THINFILM) { /* probForThinFilm(tf, hinfo, o:=i, i:=o, p), cg.hpp:1932-1949 */
    v3 const bo = i, bi = o;
    v3 const n = h->F.z;
    if (!h->front || vdot(bi, n) < 0.f || vdot(bo, n) < 0.f) return 0.f;
    v3 const hv = half_vec(bi, bo, n);
    return p * powf(vdot(bo, hv), m->alpha + 1) * (m->alpha + 1) * .5f * INV_PI * .25f;
  }
  return 0.f;
}

/* ---- the path (src/renderer.cpp:64-146) --------------------------------------------------- */

static hero trace_path(const ctx_t* c, const hero* l, const ray* r, rng_t* rng, uint32_t scatters,
                       uint32_t max_scatter, float p) {
  const lgpu_scene* sc = c->sc;
  int const K = c->K;
  hitinfo h;
  hinfo_init(&h);
  if (!isect_scene(sc, r, &h, UINT32_MAX)) return hzero();
  v3 const o = vneg(vnorm(r->u));
  v3 const n = hinfo_n(&h);
  const lgpu_material* m = &sc->materials[h.mat];
  if (m->type == LGPU_MAT_EMITTER) return spec_hero(c, m->spectrum[0], l);
  if (m->type == LGPU_MAT_DIREMITTER)
    return hscale(spec_hero(c, m->spectrum[0], l), powf(nmax(vdot(o, h.F.z), 0.f), m->specular), K);
  if (scatters > max_scatter) return hzero();
  /* sample::lights (cg.hpp:1548-1557) */
  uint64_t const li = rng_u64(rng) % (uint64_t)sc->n_lights;
  float const prob_l = 1.f / (float)sc->n_lights;
  const lgpu_light* L = &sc->lights[li];
  sinfo sl;
  sample_light(c, L, l, &h, rng, &sl);
  hero const coef = bxdf(c, m, l, sl.val, o, n, h.front);
  hero L_IS;
  for (int k = 0; k < K; k++) L_IS.v[k] = sl.mult.v[k] * coef.v[k] / (sl.prob * prob_l);
  sinfo sm;
  if (!sample_material(c, m, l, &h, o, rng, p, &sm)) return L_IS;
  ray const ir = mkray(h.p, sm.val);
  hero const Li = trace_path(c, l, &ir, rng, scatters + 1, max_scatter, p);
  hero M_IS;
  for (int k = 0; k < K; k++) M_IS.v[k] = Li.v[k] * sm.mult.v[k] / sm.prob;
  float const p_L_mati = prob_for_light(c, L, &ir) * prob_l;
  float const p_mat_Li = prob_for_material(c, m, l->v[0], &h, sl.val, o, p);
  float const p_L_i = sl.prob * prob_l;
  float const w_L = p_L_i * p_L_i / (p_L_i * p_L_i + p_mat_Li * p_mat_Li);
  float const w_mat = sm.prob * sm.prob / (sm.prob * sm.prob + p_L_mati * p_L_mati);
  hero R;
  for (int k = 0; k < K; k++) R.v[k] = M_IS.v[k] * w_mat + L_IS.v[k] * w_L;
  return R;
}

/* coefficientλ::addHeroλ (cg.hpp:306-320) */
static void add_hero(const ctx_t* c, float* v, const hero* l, const hero* s) {
  uint32_t const n = c->nb;
  for (int k = 0; k < c->K; k++) {
    uint32_t i = 0;
    for (; c->inf + (float)i * c->delta <= l->v[k] && i < n; i++) {
    }
    float const l1 = c->inf + (float)i * c->delta;
    float t = (l1 - l->v[k]) / c->delta;
    if (i == 0) t = 1.f;
    if (i == n) t = 0.f;
    if (i > 0) v[i - 1] += (1.f - t) * s->v[k];
    if (i < n) v[i] += t * s->v[k];
  }
}

void oracle_render_rows(const lgpu_scene* sc, uint32_t spp, uint32_t max_scatter, float sample_p,
                        int rng_mode, uint64_t seed, uint32_t spp_offset, uint64_t row0,
                        uint64_t row1, int fp64, float* out32, double* out64) {
  ctx_t c;
  c.sc = sc;
  c.K = (int)sc->spec.hero_k;
  c.nb = sc->spec.n_bins;
  c.inf = sc->spec.lambda_inf;
  c.sup = sc->spec.lambda_sup;
  c.delta = (c.sup - c.inf) / (float)(c.nb - 1);
  if (c.K > KMAX || c.nb > NBMAX) abort();
  uint64_t const w = sc->cam.width;
  const lgpu_camera* cam = &sc->cam;
  v3 const Fx = vload(cam->base_x), Fy = vload(cam->base_y), Fz = vload(cam->base_z);
  v3 const P = vload(cam->pos);
  int64_t const npix = (int64_t)((row1 - row0) * w);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t q = 0; q < npix; q++) {
    uint64_t const i = row0 + (uint64_t)q / w, j = (uint64_t)q % w;
    rng_t rng;
    rng.mode = rng_mode;
    if (rng_mode == ORACLE_RNG_MT19937) mt_seed(&rng.mt, i * w + j);
    float acc[NBMAX];
    double acc64[NBMAX];
    memset(acc, 0, sizeof(float) * c.nb);
    memset(acc64, 0, sizeof(double) * c.nb);
    for (uint32_t k = 0; k < spp; k++) {
      if (rng_mode == ORACLE_RNG_PCG) rng.pcg = lgpu_path_state(seed, i * w + j, (uint64_t)spp_offset + k);
      float const u = (float)j + rng_flt(&rng);
      float const v = (float)i + rng_flt(&rng);
      /* sample::camera (cg.hpp:1534-1542) */
      v3 const wij = vsub(vadd(vadd(P, vmul(Fx, -0.5f * cam->w + cam->delta * u)),
                               vmul(Fy, -0.5f * cam->h + cam->delta * v)),
                          vmul(Fz, cam->D));
      float la, lb;
      if (rng_mode == ORACLE_RNG_MT19937 && g_mt_rtl) {
        lb = rng_flt(&rng) - .5f;
        la = rng_flt(&rng) - .5f;
      } else {
        la = rng_flt(&rng) - .5f;
        lb = rng_flt(&rng) - .5f;
      }
      v3 const wkl = vadd(P, vmul(vadd(vmul(Fx, la), vmul(Fy, lb)), 2 * cam->dof));
      ray const r = mkray(wkl, vnorm(vsub(wij, wkl)));
      /* sample::spectrum (cg.hpp:1517-1531) */
      float const omega = c.sup - c.inf;
      float const hero0 = c.inf + omega * rng_flt(&rng);
      float const step = omega / (float)c.K;
      hero lam;
      for (int kk = 0; kk < c.K; kk++) {
        float x = hero0 + (float)kk * step;
        if (x > c.sup) x -= omega;
        lam.v[kk] = x;
      }
      float const prob = 1.f / omega;
      hero const Li = trace_path(&c, &lam, &r, &rng, 0, max_scatter, sample_p);
      hero const val = hdivs(Li, prob, c.K);
      if (fp64) {
        float one[NBMAX];
        memset(one, 0, sizeof(float) * c.nb);
        add_hero(&c, one, &lam, &val);
        for (uint32_t b = 0; b < c.nb; b++) acc64[b] += one[b];
      } else {
        add_hero(&c, acc, &lam, &val);
      }
    }
    size_t const o = 3 * (size_t)q;
    if (fp64) {
      double const norm = 1.0 / ((double)spp * c.K);
      double X = 0, Y = 0, Z = 0;
      for (uint32_t b = 0; b < c.nb; b++) {
        X += acc64[b] * norm * sc->spec.cmf_x[b];
        Y += acc64[b] * norm * sc->spec.cmf_y[b];
        Z += acc64[b] * norm * sc->spec.cmf_z[b];
      }
      X *= c.delta;
      Y *= c.delta;
      Z *= c.delta;
      out64[o + 0] = 3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z;
      out64[o + 1] = -0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z;
      out64[o + 2] = 0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z;
    } else {
      /* coefλ2linRGB(irradiance / float(SPP*K)) (src/renderer.cpp:52-55) */
      float const d = (float)((uint64_t)spp * (uint64_t)c.K);
      float X = 0.f, Y = 0.f, Z = 0.f;
      for (uint32_t b = 0; b < c.nb; b++) {
        float const vb = acc[b] / d;
        X += vb * sc->spec.cmf_x[b];
        Y += vb * sc->spec.cmf_y[b];
        Z += vb * sc->spec.cmf_z[b];
      }
      X = X * c.delta;
      Y = Y * c.delta;
      Z = Z * c.delta;
      out32[o + 0] = 3.2404542f * X - 1.5371385f * Y - 0.4985314f * Z;
      out32[o + 1] = -0.9692660f * X + 1.8760108f * Y + 0.0415560f * Z;
      out32[o + 2] = 0.0556434f * X - 0.2040259f * Y + 1.0572252f * Z;
    }
  }
}

/* ---- single functions, for pinning ------------------------------------------------------ */

static ctx_t unit_ctx(const lgpu_scene* sc) {
  ctx_t c;
  c.sc = sc;
  c.K = (int)sc->spec.hero_k;
  c.nb = sc->spec.n_bins;
  c.inf = sc->spec.lambda_inf;
  c.sup = sc->spec.lambda_sup;
  c.delta = (c.sup - c.inf) / (float)(c.nb - 1);
  if (c.K > KMAX || c.nb > NBMAX) abort();
  return c;
}
static hero unit_hero(const ctx_t* c, const float* lam) {
  hero l = hzero();
  for (int k = 0; k < c->K; k++) l.v[k] = lam[k];
  return l;
}
static hitinfo unit_hit(const oracle_hit* o) {
  hitinfo h;
  hinfo_init(&h);
  h.z = o->z;
  h.p = vload(o->p);
  h.F.x = vload(o->Fx);
  h.F.y = vload(o->Fy);
  h.F.z = vload(o->Fz);
  h.gn = vload(o->gn);
  h.front = o->front != 0;
  h.mat = o->mat;
  h.obj = o->obj;
  return h;
}
static void unit_put(const ctx_t* c, const hero* v, float* out) {
  for (int k = 0; k < c->K; k++) out[k] = v->v[k];
}

void oracle_unit_spectrum(const lgpu_scene* sc, uint32_t s, const float* lam, float* out) {
  ctx_t const c = unit_ctx(sc);
  hero const l = unit_hero(&c, lam);
  hero const r = spec_hero(&c, (int32_t)s, &l);
  unit_put(&c, &r, out);
}

void oracle_unit_add_hero(const lgpu_scene* sc, const float* lam, const float* v, float* out_bins) {
  ctx_t const c = unit_ctx(sc);
  hero const l = unit_hero(&c, lam), s = unit_hero(&c, v);
  memset(out_bins, 0, sizeof(float) * c.nb);
  add_hero(&c, out_bins, &l, &s);
}

void oracle_unit_bxdf(const lgpu_scene* sc, uint32_t mat, const float* lam, const float* i,
                      const float* o, const float* n, int front, float* out) {
  ctx_t const c = unit_ctx(sc);
  hero const l = unit_hero(&c, lam);
  hero const r = bxdf(&c, &sc->materials[mat], &l, vload(i), vload(o), vload(n), front);
  unit_put(&c, &r, out);
}

float oracle_unit_prob_for_material(const lgpu_scene* sc, float l0, const oracle_hit* h,
                                    const float* i, const float* o, float p) {
  ctx_t const c = unit_ctx(sc);
  hitinfo const hh = unit_hit(h);
  return prob_for_material(&c, &sc->materials[hh.mat], l0, &hh, vload(i), vload(o), p);
}

int oracle_unit_sample_material(const lgpu_scene* sc, const float* lam, const oracle_hit* h,
                                const float* o, uint64_t seed, float p, float* prob, float* dir,
                                float* mult) {
  ctx_t const c = unit_ctx(sc);
  hero const l = unit_hero(&c, lam);
  hitinfo const hh = unit_hit(h);
  rng_t rng;
  rng.mode = ORACLE_RNG_MT19937;
  mt_seed(&rng.mt, seed);
  sinfo si;
  si.prob = 0.f;
  si.val = V3(0.f, 0.f, 0.f);
  si.mult = hzero();
  int const ok = sample_material(&c, &sc->materials[hh.mat], &l, &hh, vload(o), &rng, p, &si);
  *prob = si.prob;
  dir[0] = si.val.x;
  dir[1] = si.val.y;
  dir[2] = si.val.z;
  unit_put(&c, &si.mult, mult);
  return ok;
}

void oracle_unit_sample_light(const lgpu_scene* sc, uint32_t light, const float* lam,
                              const oracle_hit* h, uint64_t seed, float* prob, float* dir,
                              float* mult) {
  ctx_t const c = unit_ctx(sc);
  hero const l = unit_hero(&c, lam);
  hitinfo const hh = unit_hit(h);
  rng_t rng;
  rng.mode = ORACLE_RNG_MT19937;
  mt_seed(&rng.mt, seed);
  sinfo si;
  si.prob = 0.f;
  si.val = V3(0.f, 0.f, 0.f);
  si.mult = hzero();
  sample_light(&c, &sc->lights[light], &l, &hh, &rng, &si);
  *prob = si.prob;
  dir[0] = si.val.x;
  dir[1] = si.val.y;
  dir[2] = si.val.z;
  unit_put(&c, &si.mult, mult);
}

float oracle_unit_prob_for_light(const lgpu_scene* sc, uint32_t light, const float* ray6) {
  ctx_t const c = unit_ctx(sc);
  ray const r = mkray(vload(ray6), vload(ray6 + 3));
  return prob_for_light(&c, &sc->lights[light], &r);
}
