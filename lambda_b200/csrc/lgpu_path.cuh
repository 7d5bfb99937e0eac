// lgpu_path.cuh — spectral MIS path tracing on the device.
//
// One path carries K hero wavelengths (the reference uses K = 16,
// cg.hpp:41).  Its geometry (hits, sampled directions, pdfs, MIS weights)
// follows the first wavelength exactly as Renderer::tracePath does
// (src/renderer.cpp:64-146); the K spectral values are evaluated in one
// fused per-wavelength loop per vertex, so no spectral temporaries are kept
// across the vertex.  The recursion of tracePath,
//     R_k = M_IS_k * w_mat + L_IS_k * w_L,   M_IS_k = R_{k+1} * mult / prob,
// becomes the forward loop
//     acc += beta * L_IS * w_L;   beta *= mult / prob * w_mat,
// with the reference's special cases kept: a vertex whose material sample
// is not generated adds L_IS without its MIS weight (src/renderer.cpp:120),
// emitters end the path with their radiance, and a path may scatter
// MAX_SCATTERINGS+1 times (src/renderer.cpp:85).
#pragma once

#include "lgpu_intersect.cuh"
#include "lgpu_rng.h"

namespace lgpu {

struct Stacks {
  StackEntry mesh[kStackCap];
  StackEntry tlas[kTlasStackCap];
};

// ---- spectra ---------------------------------------------------------------

// Lookup coordinate of wavelength l for coefficientλ::operator()
// (cg.hpp:289-297): -1 selects v[0], a huge value selects v[n-1].
__device__ __forceinline__ float lam_coord(const DevScene& S, float l) {
  if (l <= S.lambda_inf) return -1.f;
  if (l >= S.lambda_sup) return 1e30f;
  return (l - S.lambda_inf) / S.lambda_delta;
}

__device__ __forceinline__ float spec_at(const DevScene& S, int32_t s, float x) {
  const float* v = S.spectra + (size_t)s * S.n_bins;
  uint32_t const n = S.n_bins;
  if (x < 0.f) return __ldg(v);
  if (x >= 1e29f) return __ldg(v + n - 1);
  uint32_t const i = min((uint32_t)x, n - 2);
  float const t = x - (float)i;
  return (1.f - t) * __ldg(v + i) + t * __ldg(v + i + 1);
}

// k-th hero wavelength of sample::spectrum (cg.hpp:1517-1531)
__device__ __forceinline__ float hero_lambda(const DevScene& S, float hero, float step, int k) {
  float l = hero + (float)k * step;
  if (l > S.lambda_sup) l -= (S.lambda_sup - S.lambda_inf);
  return l;
}

// Film: the XYZ value of coefficientλ::addHeroλ (cg.hpp:306-320) of a single
// wavelength l with value s, dotted with the CMF tables (cg.hpp:283-288,
// 340-341) — without the final Δ factor.  The lower bin receives (1-t) and
// the upper bin t, as in the reference.
__device__ __forceinline__ void splat_xyz(const DevScene& S, float l, float s, float& X, float& Y,
                                          float& Z) {
  uint32_t const n = S.n_bins;
  float const inf = S.lambda_inf, D = S.lambda_delta;
  // i = number of grid points inf + m*Δ <= l (m < n), found from an
  // estimate and corrected with the reference's own comparison
  int i = (int)floorf((l - inf) / D) + 1;
  if (i < 0) i = 0;
  if (i > (int)n) i = (int)n;
  while (i > 0 && inf + (float)(i - 1) * D > l) i--;
  while (i < (int)n && inf + (float)i * D <= l) i++;
  float t = ((inf + (float)i * D) - l) / D;
  if (i == 0) t = 1.f;
  if (i == (int)n) t = 0.f;
  if (i > 0) {
    float const w = (1.f - t) * s;
    X += w * __ldg(S.cmf + (i - 1));
    Y += w * __ldg(S.cmf + n + (i - 1));
    Z += w * __ldg(S.cmf + 2 * n + (i - 1));
  }
  if (i < (int)n) {
    float const w = t * s;
    X += w * __ldg(S.cmf + i);
    Y += w * __ldg(S.cmf + n + i);
    Z += w * __ldg(S.cmf + 2 * n + i);
  }
}

// ---- sampling helpers -------------------------------------------------------

// stoch::CosHemi / UnifHemi (stoch.hpp:53-68); x0 is the first draw.
__device__ __forceinline__ f3 cos_hemi(float x0, float x1) {
  float const c2 = 1.f - x0;
  float const c = sqrtf(c2);
  float const s = sqrtf(1.f - c2);
  float sp, cp;
  sincosf(2.f * kPi * x1, &sp, &cp);
  return f3{s * cp, s * sp, c};
}
__device__ __forceinline__ f3 unif_hemi(float x0, float x1) {
  float const c = 1.f - x0;
  float const s = sqrtf(1.f - c * c);
  float sp, cp;
  sincosf(2.f * kPi * x1, &sp, &cp);
  return f3{s * cp, s * sp, c};
}
// sample::blinnh (cg.hpp:1790-1796)
__device__ __forceinline__ f3 blinn_h(float alpha, float x0, float x1) {
  float const c = powf(1.f - x0, 1.f / (alpha + 1.f));
  float const s = sqrtf(1.f - c * c);
  float sp, cp;
  sincosf(2.f * kPi * x1, &sp, &cp);
  return f3{s * cp, s * sp, c};
}
__device__ __forceinline__ f3 to_basis(const Basis& B, f3 v) {
  return f3{v.x * B.x.x + v.y * B.y.x + v.z * B.z.x, v.x * B.x.y + v.y * B.y.y + v.z * B.z.y,
            v.x * B.x.z + v.y * B.y.z + v.z * B.z.z};
}
__device__ __forceinline__ float fdot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 fnorm(f3 a) {
  float const l = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
  return f3{a.x / l, a.y / l, a.z / l};
}
// bra::reflect (bra.hpp:396-397): -x + 2(x·a)a
__device__ __forceinline__ f3 reflect(f3 x, f3 a) {
  float const s = 2.f * fdot(x, a);
  return f3{-x.x + s * a.x, -x.y + s * a.y, -x.z + s * a.z};
}
// the half vector of i and o, or the reference's fallback when they cancel
// (cg.hpp:951-954)
__device__ __forceinline__ f3 half_vec(f3 i, f3 o, f3 n) {
  f3 h = f3{i.x + o.x, i.y + o.y, i.z + o.z};
  float const l2 = h.x * h.x + h.y * h.y + h.z * h.z;
  if (l2 < kEps) {
    float const no = fdot(n, o);
    return fnorm(f3{n.x - no * o.x, n.y - no * o.y, n.z - no * o.z});
  }
  float const l = sqrtf(l2);
  return f3{h.x / l, h.y / l, h.z / l};
}
__device__ __forceinline__ float fmax0(float x) { return 0.f >= x ? 0.f : x; }  // nl::max(0,x)
__device__ __forceinline__ float schlick_F0(float n) {
  return (n * n - 2.f * n + 1.f) / (n * n + 2.f * n + 1.f);
}

// Uniform draws given explicitly (the shading unit probe): the sampling
// functions below take either a PCG state (uint64_t) or this.
struct XiDraws {
  const float* xi;
  uint32_t n, used;
};
using ::lgpu_flt;
__device__ __forceinline__ float lgpu_flt(XiDraws* r) {
  float const x = r->used < r->n ? r->xi[r->used] : 0.f;
  r->used++;
  return x;
}

// ---- lights -----------------------------------------------------------------

struct LightSample {
  f3 dir;
  float prob;   // p(ωi | light)
  float scale;  // λ-independent factor of mult (visibility, cos^spec, 1/d²)
};

__device__ __forceinline__ bool occluded(const DevScene& S, f3 p, f3 d, float tmax, uint32_t skip,
                                         bool ref_order, Stacks& st, TravStats& ts) {
  HitRec h;
  h.z = tmax;
  h.obj = UINT32_MAX;
  return scene_hit<true>(S, make_ray(p, d), h, skip, ref_order, st.mesh, st.tlas, ts);
}

__device__ __forceinline__ f3 col3(const float* M16, int c) {
  return f3{M16[c], M16[4 + c], M16[8 + c]};
}

// sample::light (cg.hpp:1560-1732) without its shadow ray: `scale` is the
// λ-independent factor of mult assuming the light is visible; tmax and skip
// describe the shadow ray the reference traces (for sphere lights up to the
// light's centre, cg.hpp:1696); tmax < 0 means no shadow ray (ambient).
template <class R>
__device__ __forceinline__ LightSample sample_light_unoccluded(const DevScene& S, const lgpu_light& L,
                                                               const HitInfo& H, R& rng,
                                                               float& tmax, uint32_t& skip) {
  LightSample ls;
  ls.scale = 0.f;
  ls.prob = 1.f;
  ls.dir = f3{0.f, 0.f, 1.f};
  tmax = -1.f;
  skip = UINT32_MAX;
  switch (L.type) {
    case LGPU_LIGHT_SPHERE: {  // cg.hpp:1671-1699
      f3 const pos = col3(L.T.M, 3);
      f3 const Lv = f3{pos.x - H.p.x, pos.y - H.p.y, pos.z - H.p.z};
      float const dist2 = fdot(Lv, Lv);
      float const r2 = L.size * L.size;
      float const sr = 1.f - sqrtf(fmax0(1.f - r2 / dist2));
      ls.prob = 0.5f / (kPi * sr);
      Basis const B = orthonormal_basis(Lv);
      float const x0 = lgpu_flt(&rng);
      float const ct = fmax0(1.f - x0 * sr);
      float const stt = sqrtf(1.f - ct * ct);
      float const x1 = lgpu_flt(&rng);
      float sp, cp;
      sincosf(2.f * kPi * x1, &sp, &cp);
      ls.dir = f3{B.x.x * stt * cp + B.y.x * stt * sp + B.z.x * ct,
                  B.x.y * stt * cp + B.y.y * stt * sp + B.z.y * ct,
                  B.x.z * stt * cp + B.y.z * stt * sp + B.z.z * ct};
      tmax = sqrtf(dist2);
      skip = L.obj;
      ls.scale = 1.f;
      break;
    }
    case LGPU_LIGHT_QUADDIR: {  // cg.hpp:1625-1655
      float const sx = 2.f * lgpu_flt(&rng) - 1.f;
      float const sy = 2.f * lgpu_flt(&rng) - 1.f;
      f3 const pos = col3(L.T.M, 3), c0 = col3(L.T.M, 0), c1 = col3(L.T.M, 1);
      f3 const x = f3{pos.x + sx * c0.x + sy * c1.x, pos.y + sx * c0.y + sy * c1.y,
                      pos.z + sx * c0.z + sy * c1.z};
      f3 const r = f3{x.x - H.p.x, x.y - H.p.y, x.z - H.p.z};
      f3 const w = fnorm(r);
      ls.dir = w;
      float const dist2 = fdot(r, r);
      f3 const nl = fnorm(col3(L.T.M, 2));
      float const cos_spec = powf(-fdot(w, nl), L.spec);
      float const pr = (L.spec + 1.f) * 0.5f * kInvPi * cos_spec * L.inv_area;
      ls.prob = 1e-6f >= pr ? 1e-6f : pr;
      tmax = sqrtf(dist2);
      skip = L.obj;
      ls.scale = cos_spec;
      break;
    }
    case LGPU_LIGHT_POINT: {  // cg.hpp:1580-1601
      f3 const Lv = f3{L.pos[0] - H.p.x, L.pos[1] - H.p.y, L.pos[2] - H.p.z};
      ls.dir = fnorm(Lv);
      float const dist = sqrtf(fdot(Lv, Lv));
      tmax = dist;
      ls.scale = 1.f / (dist * dist);
      break;
    }
    case LGPU_LIGHT_DIR: {  // cg.hpp:1604-1621
      ls.dir = f3{-L.dir[0], -L.dir[1], -L.dir[2]};
      tmax = kFltMax;
      ls.scale = 1.f;
      break;
    }
    default: {  // ambient, cg.hpp:1560-1577
      float const x0 = lgpu_flt(&rng);
      float const x1 = lgpu_flt(&rng);
      f3 d = unif_hemi(x0, x1);
      if (!H.front) d.z = -d.z;
      ls.dir = to_basis(H.F, d);
      ls.prob = 0.5f * kInvPi;
      ls.scale = 1.f;
      break;
    }
  }
  return ls;
}

// sample::light (cg.hpp:1560-1732) including the shadow ray
__device__ __forceinline__ LightSample sample_light(const DevScene& S, const lgpu_light& L,
                                                    const HitInfo& H, uint64_t& rng, bool ref_order,
                                                    Stacks& st, TravStats& ts, uint32_t& rays) {
  float tmax;
  uint32_t skip;
  LightSample ls = sample_light_unoccluded(S, L, H, rng, tmax, skip);
  if (tmax >= 0.f) {
    rays++;
    if (occluded(S, H.p, ls.dir, tmax, skip, ref_order, st, ts)) ls.scale = 0.f;
  }
  return ls;
}

// sample::probForLight (cg.hpp:1735-1747) for the ray (p, d)
__device__ __forceinline__ float prob_for_light(const DevScene& S, const lgpu_light& L, f3 p, f3 d) {
  if (L.type == LGPU_LIGHT_SPHERE) {  // cg.hpp:1702-1714
    Ray const w = make_ray(p, d);
    DevObject ob;
    for (int q = 0; q < 12; q++) ob.M_inv[q] = L.T.M_inv[q];
    Ray const l = to_local(ob, w);
    float t;
    if (!sphere_test(l, kFltMax, t)) return 0.f;
    f3 const pl = ray_at(l, t);
    f3 const n = normalized(normal_to_world(L.T.M_inv, pl));
    if (!(dot3(n, w.u) < 0.f)) return 0.f;
    f3 const pos = col3(L.T.M, 3);
    f3 const Lv = f3{pos.x - p.x, pos.y - p.y, pos.z - p.z};
    float const dist2 = fdot(Lv, Lv);
    float const sr = 1.f - sqrtf(fmax0(1.f - L.size * L.size / dist2));
    return 0.5f / (kPi * sr);
  }
  if (L.type == LGPU_LIGHT_QUADDIR) {  // cg.hpp:1657-1668
    Ray const w = make_ray(p, d);
    DevObject ob;
    for (int q = 0; q < 12; q++) ob.M_inv[q] = L.T.M_inv[q];
    Ray const l = to_local(ob, w);
    float t;
    f3 x;
    if (!plane_test(l, kFltMax, t, x)) return 0.f;
    f3 const Fz = normalized(normal_to_world(L.T.M_inv, mk(0.f, 0.f, 1.f)));
    if (!(dot3(w.u, Fz) < 0.f)) return 0.f;
    f3 const un = fnorm(d);
    float const ct = -(un.x * Fz.x + un.y * Fz.y + un.z * Fz.z);
    float const pr = (L.spec + 1.f) * 0.5f * kInvPi * powf(ct, L.spec) * L.inv_area;
    return 1e-6f >= pr ? 1e-6f : pr;
  }
  if (L.type == LGPU_LIGHT_AMBIENT) return 0.5f * kInvPi;
  return 0.f;
}

// ---- materials ---------------------------------------------------------------

// λ-independent part of BxDFcosθ(λ, mat, i, o, n, front) (cg.hpp:1088-1102)
struct BsdfScalars {
  int kind;    // 0: zero, 1: lambertian, 2: blinn reflect side, 3: blinn transmit side, 4: thinfilm
  float a;     // lambertian/blinn: max(0, cos_i); thinfilm: cos_i (i·h)
  float b;     // blinn: pow(1-cos_o, 5); thinfilm: pow(1-cos_i, 5)
  float c;     // blinn: pow(h·n, α) or pow(|ht·n|, α); thinfilm: pow(h·n, α)
  float lnhn;  // log of the |cosine| raised to α in c (for d/dα)
};

__device__ __forceinline__ BsdfScalars bsdf_scalars(const DevScene& S, const DevMaterial& m,
                                                    float x0, f3 i, f3 o, f3 n, bool front) {
  BsdfScalars r;
  r.kind = 0;
  r.a = r.b = r.c = r.lnhn = 0.f;
  if (m.type == LGPU_MAT_LAMBERTIAN) {  // cg.hpp:921-926
    r.kind = 1;
    r.a = fmax0(fdot(i, n));
  } else if (m.type == LGPU_MAT_BLINN) {  // cg.hpp:944-967
    float const cos_i = fdot(i, n), cos_o = fdot(o, n);
    r.a = fmax0(cos_i);
    r.b = powf(1.f - cos_o, 5.f);
    if (cos_i * cos_o > 0.f) {
      r.kind = 2;
      f3 const h = half_vec(i, o, n);
      float const hn = fdot(h, n);
      r.c = powf(hn, m.alpha);
      r.lnhn = logf(fabsf(hn));
    } else {
      r.kind = 3;
      float const ior0 = spec_at(S, m.spectrum[4], x0);
      float const eta0 = front ? 1.f / ior0 : ior0;
      f3 const ht = fnorm(f3{i.x + eta0 * o.x, i.y + eta0 * o.y, i.z + eta0 * o.z});
      float const hn = fabsf(fdot(ht, n));
      r.c = powf(hn, m.alpha);
      r.lnhn = logf(hn);
    }
  } else if (m.type == LGPU_MAT_THINFILM) {  // cg.hpp:1032-1051
    if (front && !(fdot(i, n) < 0.f) && !(fdot(o, n) < 0.f)) {
      r.kind = 4;
      f3 const h = half_vec(i, o, n);
      r.a = fdot(i, h);
      r.b = powf(1.f - r.a, 5.f);
      float const hn = fdot(h, n);
      r.c = powf(hn, m.alpha);
      r.lnhn = logf(fabsf(hn));
    }
  }
  return r;
}

// thinfilm::BRDFcosθ at one wavelength (cg.hpp:1001-1051)
__device__ __forceinline__ float thinfilm_k(const DevScene& S, const DevMaterial& m, float x, float l,
                                            float cos_i, float pow5, float pow_hn) {
  float const n1 = spec_at(S, m.spectrum[0], x);
  float const n2 = spec_at(S, m.spectrum[1], x);
  float const n01 = 1.f / n1;
  float const cos_l = sqrtf(1.f - n01 * n01) * (1.f - cos_i * cos_i);
  float const cos_d = cosf(4.f * kPi * n1 * m.d * cos_l / l);
  float const a01 = (1.f - n1), b01 = (1.f + n1);
  float const R0_01 = a01 * a01 / (b01 * b01);
  float const a12 = (n1 - n2), b12 = (n1 + n2);
  float const R0_12 = a12 * a12 / (b12 * b12);
  float const R01 = R0_01 + (1.f - R0_01) * pow5;
  float const R12 = R0_12 + (1.f - R0_12) * pow5;
  float const Ravg = 2.f * sqrtf(R01 * R12);
  float const Rt = (R01 + R12 + Ravg * cos_d) / (1.f + R01 * R12 + Ravg * cos_d);
  return (m.alpha + 2.f) * 0.125f * kInvPi * Rt * pow_hn;
}

// BxDFcosθ at wavelength l (lookup coordinate x) from its scalars
__device__ __forceinline__ float bsdf_k(const DevScene& S, const DevMaterial& m, const BsdfScalars& r,
                                        float x, float l, bool front) {
  switch (r.kind) {
    case 1:
      return spec_at(S, m.spectrum[0], x) * kInvPi * r.a;
    case 2:
    case 3: {
      float const ior = spec_at(S, m.spectrum[4], x);
      float const eta = front ? 1.f / ior : ior;
      float const F0 = schlick_F0(eta);
      float const F = F0 + (1.f - F0) * r.b;
      float const g = (m.alpha + 2.f) * 0.125f * kInvPi * r.c;
      if (r.kind == 2)
        return spec_at(S, m.spectrum[0], x) * kInvPi * r.a +
               (spec_at(S, m.spectrum[1], x) + F * spec_at(S, m.spectrum[2], x)) * g;
      return spec_at(S, m.spectrum[2], x) * (1.f - F) * g;
    }
    case 4:
      return thinfilm_k(S, m, x, l, r.a, r.b, r.c);
  }
  return 0.f;
}

// Result of sample::materiali (cg.hpp:1953-1968): direction, pdf and what is
// needed to evaluate its BxDFcosθ per wavelength.
struct MatSample {
  bool ok;
  f3 dir;
  float prob;
  int lobe;  // 1 lambert/blinn-diffuse (a=max(0,cos)), 2 blinn reflect, 3 blinn transmit, 4 thinfilm
  float a, b, c;
  float cos_oh;  // blinn: o·h, for the per-wavelength total-internal-reflection test
  float lnhn;    // log of the |cosine| raised to α in c (for d/dα)
  float dlnprob; // d ln(prob) / dα: 0 for the lobes whose pdf does not depend on α
};

template <class R>
__device__ __forceinline__ MatSample sample_material(const DevScene& S, const DevMaterial& m, float x0,
                                                     const HitInfo& H, f3 o, float p, R& rng) {
  MatSample ms;
  ms.ok = false;
  ms.prob = 0.f;
  ms.lobe = 0;
  ms.a = ms.b = ms.c = ms.cos_oh = ms.lnhn = ms.dlnprob = 0.f;
  ms.dir = f3{0.f, 0.f, 1.f};
  f3 const n = H.front ? H.F.z : neg3(H.F.z);
  if (m.type == LGPU_MAT_LAMBERTIAN) {  // cg.hpp:1755-1777
    float const xi = lgpu_flt(&rng);
    if (xi > p) return ms;
    float const u0 = lgpu_flt(&rng), u1 = lgpu_flt(&rng);
    f3 d = cos_hemi(u0, u1);
    if (!H.front) d.z = -d.z;
    f3 const i = to_basis(H.F, d);
    ms.ok = true;
    ms.dir = i;
    ms.prob = p * fabsf(d.z) * kInvPi;
    ms.lobe = 1;
    ms.a = fmax0(fdot(i, n));
    return ms;
  }
  if (m.type == LGPU_MAT_BLINN) {  // cg.hpp:1799-1862
    float const lobe = lgpu_flt(&rng);
    if (lobe >= p) return ms;
    float const pp_d = p * m.p_d, pp_spec = p * m.p_spec;
    if (lobe < pp_spec) {
      float const ior0 = spec_at(S, m.spectrum[4], x0);
      float const eta0 = H.front ? 1.f / ior0 : ior0;
      float const u0 = lgpu_flt(&rng), u1 = lgpu_flt(&rng);
      f3 w = blinn_h(m.alpha, u0, u1);
      if (!H.front) w.z = -w.z;
      f3 const h = to_basis(H.F, w);
      float const cos_oh = fdot(o, h);
      // transmit() (cg.hpp:500-513) for the first wavelength
      float const ct2 = 1.f - eta0 * eta0 * (1.f - cos_oh * cos_oh);
      float F = 1.f;
      f3 iT = f3{0.f, 0.f, 0.f};
      if (!(ct2 < 0.f)) {
        float const F0 = schlick_F0(eta0);
        F = F0 + (1.f - F0) * powf(1.f - cos_oh, 5.f);
        float const k = sqrtf(ct2) - eta0 * cos_oh;
        iT = f3{-eta0 * o.x - k * h.x, -eta0 * o.y - k * h.y, -eta0 * o.z - k * h.z};
        if (iT.x == 0.f && iT.y == 0.f && iT.z == 0.f) F = 1.f;
      }
      // blinn::fresnelSplit (cg.hpp:951-960) on F[0]
      float p_r = m.w_r + F * m.w_t, p_t = (1.f - F) * m.w_t;
      float const tot = p_r + p_t;
      if (tot == 0.f) {
        p_r = 1.f;
        p_t = 0.f;
      } else {
        p_r /= tot;
        p_t /= tot;
      }
      float const hp = powf(fabsf(w.z), m.alpha + 1.f) * (m.alpha + 1.f) * 0.5f * kInvPi;
      ms.ok = true;
      ms.cos_oh = cos_oh;
      ms.c = powf(w.z, m.alpha);
      ms.lnhn = logf(fabsf(w.z));
      // hp = (α+1)/(2π) |h·n|^(α+1)
      ms.dlnprob = 1.f / (m.alpha + 1.f) + ms.lnhn;
      if (lobe < pp_spec * p_r) {
        ms.prob = pp_spec * p_r * hp * 0.25f;
        ms.dir = reflect(o, h);
        ms.lobe = 2;
      } else {
        ms.prob = pp_spec * p_t * hp * 0.25f;
        ms.dir = iT;
        ms.lobe = 3;
      }
      return ms;
    }
    if (lobe < pp_spec + pp_d) {
      float const u0 = lgpu_flt(&rng), u1 = lgpu_flt(&rng);
      f3 d = cos_hemi(u0, u1);
      if (!H.front) d.z = -d.z;
      ms.ok = true;
      ms.dir = to_basis(H.F, d);
      ms.prob = pp_d * (fabsf(d.z) * kInvPi);
      ms.lobe = 1;
      ms.a = fmax0(d.z);
      return ms;
    }
    return ms;
  }
  if (m.type == LGPU_MAT_THINFILM) {  // cg.hpp:1905-1929
    f3 const nz = H.F.z;
    if (!H.front || fdot(o, nz) < 0.f) return ms;
    float const lobe = lgpu_flt(&rng);
    if (lobe >= p) return ms;
    float const u0 = lgpu_flt(&rng), u1 = lgpu_flt(&rng);
    f3 const w = blinn_h(m.alpha, u0, u1);
    f3 const h = to_basis(H.F, w);
    f3 const i = reflect(o, h);
    ms.ok = true;
    ms.dir = i;
    ms.prob = p * powf(fdot(nz, h), m.alpha + 1.f) * (m.alpha + 1.f) * 0.5f * kInvPi * 0.25f;
    ms.dlnprob = 1.f / (m.alpha + 1.f) + logf(fdot(nz, h));
    // its mult is thinfilm::BRDFcosθ(l, i, o, F.z, front)
    ms.lobe = 0;
    if (!(fdot(i, nz) < 0.f) && !(fdot(o, nz) < 0.f)) {
      ms.lobe = 4;
      f3 const hh = half_vec(i, o, nz);
      ms.a = fdot(i, hh);
      ms.b = powf(1.f - ms.a, 5.f);
      float const hn = fdot(hh, nz);
      ms.c = powf(hn, m.alpha);
      ms.lnhn = logf(fabsf(hn));
    }
    return ms;
  }
  return ms;
}

// mult of the material sample at one wavelength
__device__ __forceinline__ float mat_mult_k(const DevScene& S, const DevMaterial& m, const MatSample& ms,
                                            float x, float l, bool front) {
  switch (ms.lobe) {
    case 1:  // lambertian albedo or blinn Kd, both spectrum[0]
      return spec_at(S, m.spectrum[0], x) * kInvPi * ms.a;
    case 2:
    case 3: {
      float const ior = spec_at(S, m.spectrum[4], x);
      float const eta = front ? 1.f / ior : ior;
      float F = 1.f;
      float const ct2 = 1.f - eta * eta * (1.f - ms.cos_oh * ms.cos_oh);
      if (!(ct2 < 0.f)) {
        float const F0 = schlick_F0(eta);
        F = F0 + (1.f - F0) * powf(1.f - ms.cos_oh, 5.f);
      }
      float const g = (m.alpha + 2.f) * 0.125f * kInvPi * ms.c;
      if (ms.lobe == 2) return (spec_at(S, m.spectrum[1], x) + F * spec_at(S, m.spectrum[2], x)) * g;
      return spec_at(S, m.spectrum[2], x) * (1.f - F) * g;
    }
    case 4:
      return thinfilm_k(S, m, x, l, ms.a, ms.b, ms.c);
  }
  return 0.f;
}

// sample::probForMateriali (cg.hpp:1971-1985) as the reference calls it
// (src/renderer.cpp:136-137): probForBlinn and probForThinFilm declare
// (o, i) where the call passes (i, o), so inside them `o` is the light
// direction and `i` the view direction.
// With dlog, also d ln(prob) / dα (0 where the pdf does not depend on α),
// for the path-replay adjoint; the returned pdf is the same either way.
__device__ __forceinline__ float prob_for_material(const DevScene& S, const DevMaterial& m, float x0,
                                                   const HitInfo& H, f3 wl, f3 o, float p,
                                                   float* dlog = nullptr) {
  if (dlog) *dlog = 0.f;
  f3 const n = H.front ? H.F.z : neg3(H.F.z);
  if (m.type == LGPU_MAT_LAMBERTIAN) {  // cg.hpp:1780-1787
    float const ci = fdot(wl, n);
    if (ci < 0.f || fdot(o, n) < 0.f) return 0.f;
    return p * ci * kInvPi;
  }
  if (m.type == LGPU_MAT_BLINN) {  // cg.hpp:1865-1902 with o := wl, i := o
    f3 const bo = wl, bi = o;
    float const iorv = spec_at(S, m.spectrum[4], x0);
    float const ior = H.front ? 1.f / iorv : iorv;
    float const cos_in = fdot(bi, n), cos_on = fdot(bo, n);
    bool const refl = cos_in * cos_on > 0.f;
    f3 h;
    if (refl) h = half_vec(bi, bo, n);
    else h = neg3(fnorm(f3{bi.x + ior * bo.x, bi.y + ior * bo.y, bi.z + ior * bo.z}));
    float const cos_o = fabsf(fdot(bo, h));
    float const F0 = schlick_F0(ior);
    float const F = F0 + (1.f - F0) * powf(1.f - cos_o, 5.f);
    float p_r = m.w_r + F * m.w_t, p_t = (1.f - F) * m.w_t;
    float const tot = p_r + p_t;
    if (tot == 0.f) {
      p_r = 1.f;
      p_t = 0.f;
    } else {
      p_r /= tot;
      p_t /= tot;
    }
    float const hn = fdot(h, n);
    float const hp = powf(fabsf(hn), m.alpha + 1.f) * (m.alpha + 1.f) * 0.5f * kInvPi;
    if (refl) {
      float const spec = m.p_spec * p_r * hp * 0.25f;
      float const tot_p = p * (m.p_d * (fabsf(cos_in) * kInvPi) + spec);
      if (dlog && tot_p > 0.f) *dlog = p * spec * (1.f / (m.alpha + 1.f) + logf(fabsf(hn))) / tot_p;
      return tot_p;
    }
    float const c2 = 1.f - ior * ior * (1.f - cos_o * cos_o);
    if (c2 < 0.f) return 0.f;
    if (dlog) *dlog = 1.f / (m.alpha + 1.f) + logf(fabsf(hn));
    return p * m.p_spec * p_t * hp * 0.25f;
  }
  if (m.type == LGPU_MAT_THINFILM) {  // cg.hpp:1932-1949 with o := wl, i := o
    f3 const nz = H.F.z;
    f3 const bo = wl, bi = o;
    if (!H.front || fdot(bi, nz) < 0.f || fdot(bo, nz) < 0.f) return 0.f;
    f3 const h = half_vec(bi, bo, nz);
    if (dlog) *dlog = 1.f / (m.alpha + 1.f) + logf(fdot(bo, h));
    return p * powf(fdot(bo, h), m.alpha + 1.f) * (m.alpha + 1.f) * 0.5f * kInvPi * 0.25f;
  }
  return 0.f;
}

// ---- one path -----------------------------------------------------------------

struct PathCounters {
  uint32_t rays;
  TravStats ts;
};

// Renderer::tracePath (src/renderer.cpp:64-146) for the camera ray r with
// hero wavelengths (hero, step); accumulates the path's radiance per
// wavelength into acc[K].
template <int K>
__device__ __forceinline__ void trace_path(const DevScene& S, Ray r, float hero, float step,
                                           uint32_t max_scatter, float p, bool ref_order,
                                           uint64_t& rng, float (&acc)[K], Stacks& st,
                                           PathCounters& pc) {
  float beta[K];
  float xk[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    beta[k] = 1.f;
    acc[k] = 0.f;
    xk[k] = lam_coord(S, hero_lambda(S, hero, step, k));
  }
  for (uint32_t scatters = 0;; scatters++) {
    HitRec h;
    h.z = kFltMax;
    h.obj = UINT32_MAX;
    pc.rays++;
    if (!scene_hit<false>(S, r, h, UINT32_MAX, ref_order, st.mesh, st.tlas, pc.ts)) return;
    HitInfo const H = finalize_hit(S, r, h);
    f3 const un = fnorm(r.u);
    f3 const o = f3{-un.x, -un.y, -un.z};
    f3 const n = H.front ? H.F.z : neg3(H.F.z);
    const DevMaterial& m = S.mats[H.mat];
    if (m.type == LGPU_MAT_EMITTER || m.type == LGPU_MAT_DIREMITTER) {
      float g = 1.f;
      if (m.type == LGPU_MAT_DIREMITTER) {
        float const c = fdot(o, H.F.z);
        g = powf(c >= 0.f ? c : 0.f, m.specular);
      }
#pragma unroll
      for (int k = 0; k < K; k++) acc[k] += beta[k] * (spec_at(S, m.spectrum[0], xk[k]) * g);
      return;
    }
    if (scatters > max_scatter) return;

    // light importance sample (src/renderer.cpp:87-107)
    uint32_t const li = (uint32_t)(lgpu_u64(&rng) % (uint64_t)S.n_lights);
    float const prob_l = 1.f / (float)S.n_lights;
    const lgpu_light& L = S.lights[li];
    LightSample const ls = sample_light(S, L, H, rng, ref_order, st, pc.ts, pc.rays);
    BsdfScalars const bl = bsdf_scalars(S, m, xk[0], ls.dir, o, n, H.front);

    // material importance sample (src/renderer.cpp:109-120)
    MatSample const ms = sample_material(S, m, xk[0], H, o, p, rng);
    float w_L = 1.f, w_mat = 0.f;
    if (ms.ok) {
      // MIS weights, power heuristic β=2 (src/renderer.cpp:133-143)
      float const p_L_mati = prob_for_light(S, L, H.p, ms.dir) * prob_l;
      float const p_mat_Li = prob_for_material(S, m, xk[0], H, ls.dir, o, p);
      float const p_L_i = ls.prob * prob_l;
      w_L = p_L_i * p_L_i / (p_L_i * p_L_i + p_mat_Li * p_mat_Li);
      w_mat = ms.prob * ms.prob / (ms.prob * ms.prob + p_L_mati * p_L_mati);
    }
    float const lis_scale = ls.scale / (ls.prob * prob_l) * w_L;
    float const m_scale = ms.ok ? w_mat / ms.prob : 0.f;
#pragma unroll
    for (int k = 0; k < K; k++) {
      float const l = hero_lambda(S, hero, step, k);
      float const coef = bsdf_k(S, m, bl, xk[k], l, H.front);
      float const rad = spec_at(S, L.spectrum, xk[k]);
      acc[k] += beta[k] * (rad * coef * lis_scale);
      if (ms.ok) beta[k] *= mat_mult_k(S, m, ms, xk[k], l, H.front) * m_scale;
    }
    if (!ms.ok) return;
    r = make_ray(H.p, ms.dir);
  }
}

}  // namespace lgpu
