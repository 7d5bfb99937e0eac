// ref_harness.cpp — TEST INFRASTRUCTURE ONLY (oracle).
//
// A C interface over the reference renderer, compiled from the reference's
// own sources where they lie (src/renderer.cpp, lib/numli/*.hpp, the
// vendored loaders) by oracle/Makefile into oracle/_ref/libref*.so.  Tests
// and the CPU-baseline leg of bench.py load it through ctypes to
//   - load .nls scenes with the reference loader (cg.hpp:2455-2470),
//   - export them through the drop-in flattener (lgpu_flatten.hpp),
//   - run intersect::scene on ray sets (cg.hpp:1469-1489),
//   - render with Renderer::render / Renderer::tracePath
//     (src/renderer.cpp:14-146), optionally over a band of rows and with
//     FP64 accumulation,
//   - evaluate single reference functions (materials, pdfs, light and
//     material sampling, spectra, tone mapping) for known-answer tests.
// Nothing in the product links or loads this file.
#include <omp.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "lgpu_flatten.hpp"
#include "renderer.hpp"

using namespace nl::cg;
using nl::ℝ3;

namespace {

struct ref_scene {
  nl::cg::scene sc;
  lgpu_host::flat_scene flat;
};

ℝ3 v3(float const* p) { return ℝ3{p[0], p[1], p[2]}; }
void put3(ℝ3 const& v, float* out) {
  out[0] = v[0];
  out[1] = v[1];
  out[2] = v[2];
}

// hit record exchanged with tests (mirrors hitinfo, cg.hpp:1138-1149)
struct ref_hitinfo {
  float z;
  float p[3];
  float Fx[3], Fy[3], Fz[3];
  float gn[3];
  uint32_t front, mat, obj;
};

hitinfo to_hinfo(ref_hitinfo const& h) {
  hitinfo x;
  x.z = h.z;
  x.p = v3(h.p);
  x.F = basis(v3(h.Fx), v3(h.Fy), v3(h.Fz));
  x.gn = v3(h.gn);
  x.front = h.front != 0;
  x.mat = h.mat;
  x.obj = h.obj;
  return x;
}

heroλ hero_from(float const* l) {
  float v[HERO_SAMPLES];
  for (int k = 0; k < HERO_SAMPLES; k++) v[k] = l[k];
  return heroλ(v);
}

void hero_out(heroλ const& x, float* out) {
  for (int k = 0; k < HERO_SAMPLES; k++) out[k] = x[k];
}

coefficientλ<Nλ>* table(int which) {
  switch (which) {
    case 0: return &CMF_X;
    case 1: return &CMF_Y;
    case 2: return &CMF_Z;
    case 3: return &bt_709_r;
    case 4: return &bt_709_g;
    case 5: return &bt_709_b;
  }
  return nullptr;
}

}  // namespace

extern "C" {

int ref_n_bins() { return Nλ; }
int ref_hero_samples() { return HERO_SAMPLES; }
// coefficientλ's compiled-in wavelength range (cg.hpp:244-245)
void ref_lambda_range(float* out2) {
  coefficientλ<Nλ> const probe(0.f);
  out2[0] = probe.inf;
  out2[1] = probe.sup;
}

// The reference fills CMF_X/Y/Z and the BT.709 basis at static
// initialisation from relative paths (cg.hpp:329-337).  These two calls read
// and overwrite the six 80-bin tables.
void ref_get_tables(float* out6xN) {
  for (int t = 0; t < 6; t++)
    for (uint32_t i = 0; i < Nλ; i++) out6xN[t * Nλ + i] = table(t)->v[i];
}
void ref_set_tables(float const* in6xN) {
  for (int t = 0; t < 6; t++)
    for (uint32_t i = 0; i < Nλ; i++) table(t)->v[i] = in6xN[t * Nλ + i];
}

// coefficientλ<Nλ>(sampledλ) (cg.hpp:252-272) on (l, v) pairs.
void ref_coef_from_samples(float const* l, float const* v, uint64_t n,
                           float* out) {
  sampledλ s("");  // empty: the file does not exist
  s.l.assign(l, l + n);
  s.v.assign(v, v + n);
  coefficientλ<Nλ> c(s);
  for (uint32_t i = 0; i < Nλ; i++) out[i] = c.v[i];
}

void* ref_load(char const* nls_path) {
  auto* r = new ref_scene;
  bool ok = false;
  try {
    ok = load::loadNLS(r->sc, nls_path);
  } catch (...) {
    ok = false;
  }
  if (!ok) {
    delete r;
    return nullptr;
  }
  lgpu_host::flatten(r->sc, r->flat);
  return r;
}

void ref_free(void* h) { delete static_cast<ref_scene*>(h); }

lgpu_scene const* ref_export(void* h) {
  return &static_cast<ref_scene*>(h)->flat.scene;
}

// Camera settings as loaded (cg.hpp:2039-2069).
void ref_camera(void* h, uint64_t* wh) {
  auto* r = static_cast<ref_scene*>(h);
  wh[0] = r->sc.cam.width;
  wh[1] = r->sc.cam.height;
}

// intersect::scene on n rays (ray = p xyz, u xyz); hits as lgpu_hit with
// face = UINT32_MAX (hitinfo has no face field).
void ref_intersect(void* h, float const* rays, uint64_t n, lgpu_hit* out) {
  auto* r = static_cast<ref_scene*>(h);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < int64_t(n); i++) {
    float const* q = rays + 6 * i;
    ray const rr(v3(q), v3(q + 3));
    hitinfo hinfo;
    lgpu_hit& o = out[i];
    std::memset(&o, 0, sizeof(o));
    o.face = UINT32_MAX;
    if (intersect::scene(r->sc, rr, hinfo)) {
      o.t = hinfo.z;
      o.obj = hinfo.obj;
      o.mat = hinfo.mat;
      put3(hinfo.p, o.p);
      put3(hinfo.F.z, o.n);
      put3(hinfo.gn, o.gn);
      o.front = hinfo.front ? 1u : 0u;
    } else {
      o.t = hinfo.z;
      o.obj = UINT32_MAX;
      o.mat = UINT32_MAX;
    }
  }
}

// Shadow-style query: intersect::scene with hinfo.z preset and an object to
// skip (cg.hpp:1469-1489 with `skip`).
void ref_occluded(void* h, float const* rays, float const* tmax,
                  uint32_t const* skip, uint64_t n, uint8_t* out) {
  auto* r = static_cast<ref_scene*>(h);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < int64_t(n); i++) {
    float const* q = rays + 6 * i;
    hitinfo hinfo;
    hinfo.z = tmax[i];
    out[i] = intersect::scene(r->sc, ray(v3(q), v3(q + 3)), hinfo, skip[i]) ? 1 : 0;
  }
}

// Renderer::render (src/renderer.cpp:14-61), unchanged.
void ref_render(void* h, uint64_t spp, uint64_t max_scatter, float sample_p,
                float* out_rgb) {
  auto* r = static_cast<ref_scene*>(h);
  Renderer rd;
  rd.SPP = spp;
  rd.MAX_SCATTERINGS = max_scatter;
  rd.SAMPLE_P = sample_p;
  rendering buf;
  rd.render(r->sc, buf);
  size_t const N = buf.img.width * buf.img.height;
  for (size_t i = 0; i < N; i++) {
    out_rgb[3 * i + 0] = buf.img.data[i].c[0];
    out_rgb[3 * i + 1] = buf.img.data[i].c[1];
    out_rgb[3 * i + 2] = buf.img.data[i].c[2];
  }
}

// The pixel loop of Renderer::render (src/renderer.cpp:27-56) over the image
// rows [row0, row1) only — the same per-pixel seeding, sampling calls and
// tracePath — so that a bounded band of a large image can be timed or used
// as an oracle.  The band is NOT flipped: out holds (row1-row0)*w*3 values
// and band row k is scene row i = row0+k, which Renderer::render stores at
// buffer row h-1-i (src/renderer.cpp:54).  With fp64 != 0
// the per-sample 80-bin splats are accumulated in double precision and the
// colour conversion is done in double (out64 used instead of out32).
// ref_render_rows_seeded seeds pixel (i, j) with seed_base + i*w + j
// instead: seed_base = w*h gives every pixel a stream disjoint from the
// reference's own render, for an independent oracle image.
void ref_render_rows_seeded(void* h, uint64_t spp, uint64_t max_scatter,
                            float sample_p, uint64_t row0, uint64_t row1,
                            int fp64, uint64_t seed_base, float* out32,
                            double* out64) {
  auto* r = static_cast<ref_scene*>(h);
  scene const& sc = r->sc;
  Renderer rd;
  rd.SPP = spp;
  rd.MAX_SCATTERINGS = max_scatter;
  rd.SAMPLE_P = sample_p;
  uint64_t const w = sc.cam.width;
  coefficientλ<Nλ> sample_spec(0.f);
  float const Δ = sample_spec.Δ;
#pragma omp parallel for collapse(2) schedule(runtime)
  for (uint64_t i = row0; i < row1; i++)
    for (uint64_t j = 0; j < w; j++) {
      nl::RNG rng(seed_base + i * w + j);
      coefficientλ<Nλ> acc(0.f);
      double acc64[Nλ] = {0.0};
      for (uint64_t k = 0; k < spp; k++) {
        sample::info<ray> si;
        nl::ℝ2 const uv = {float(j + rng.flt()), float(i + rng.flt())};
        sample::camera(sc.cam, uv, si, rng);
        sample::info<heroλ> si_λ;
        sample::spectrum(sample_spec, si_λ, rng);
        heroλ const Li = rd.tracePath(sc, si_λ.val, si.val, rng, 0);
        if (fp64) {
          coefficientλ<Nλ> one(0.f);
          one.addHeroλ(si_λ.val, Li / si_λ.prob);
          for (uint32_t b = 0; b < Nλ; b++) acc64[b] += one.v[b];
        } else {
          acc.addHeroλ(si_λ.val, Li / si_λ.prob);
        }
      }
      uint64_t const o = (i - row0) * w + j;
      if (fp64) {
        double const norm = 1.0 / double(spp * HERO_SAMPLES);
        double X = 0, Y = 0, Z = 0;
        for (uint32_t b = 0; b < Nλ; b++) {
          X += acc64[b] * norm * CMF_X.v[b];
          Y += acc64[b] * norm * CMF_Y.v[b];
          Z += acc64[b] * norm * CMF_Z.v[b];
        }
        X *= Δ;
        Y *= Δ;
        Z *= Δ;
        out64[3 * o + 0] = 3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z;
        out64[3 * o + 1] = -0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z;
        out64[3 * o + 2] = 0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z;
      } else {
        linRGB const c = coefλ2linRGB(acc / float(spp * HERO_SAMPLES));
        out32[3 * o + 0] = c.c[0];
        out32[3 * o + 1] = c.c[1];
        out32[3 * o + 2] = c.c[2];
      }
    }
}

void ref_render_rows(void* h, uint64_t spp, uint64_t max_scatter,
                     float sample_p, uint64_t row0, uint64_t row1, int fp64,
                     float* out32, double* out64) {
  ref_render_rows_seeded(h, spp, max_scatter, sample_p, row0, row1, fp64, 0,
                         out32, out64);
}

// Renderer::tracePath (src/renderer.cpp:64-146) for one path with an RNG
// seeded by `seed`.
void ref_trace_path(void* h, float const* lam, float const* ray6,
                    uint64_t seed, uint64_t max_scatter, float sample_p,
                    float* out) {
  auto* r = static_cast<ref_scene*>(h);
  Renderer rd;
  rd.MAX_SCATTERINGS = max_scatter;
  rd.SAMPLE_P = sample_p;
  nl::RNG rng(seed);
  hero_out(rd.tracePath(r->sc, hero_from(lam), ray(v3(ray6), v3(ray6 + 3)),
                        rng, 0),
           out);
}

// RNG (stoch.hpp:30-47)
void ref_rng_flt(uint64_t seed, uint64_t n, float* out) {
  nl::RNG rng(seed);
  for (uint64_t i = 0; i < n; i++) out[i] = rng.flt();
}
void ref_rng_u64(uint64_t seed, uint64_t n, uint64_t* out) {
  nl::RNG rng(seed);
  for (uint64_t i = 0; i < n; i++) out[i] = rng.uint64();
}
// interleaved draws: kinds[i] = 0 → flt, 1 → uint64 (stored as double bits)
void ref_rng_mixed(uint64_t seed, uint64_t n, uint8_t const* kinds,
                   float* out_f, uint64_t* out_u) {
  nl::RNG rng(seed);
  for (uint64_t i = 0; i < n; i++) {
    if (kinds[i]) out_u[i] = rng.uint64();
    else out_f[i] = rng.flt();
  }
}

// Camera ray for uv with the lens draws from an RNG seeded by `seed`
// (cg.hpp:1534-1542).
void ref_camera_ray(void* h, float u, float v, uint64_t seed, float* out6) {
  auto* r = static_cast<ref_scene*>(h);
  nl::RNG rng(seed);
  sample::info<ray> si;
  nl::ℝ2 const uv = {u, v};
  sample::camera(r->sc.cam, uv, si, rng);
  put3(si.val.p, out6);
  put3(si.val.u, out6 + 3);
}

// Hero wavelengths from an RNG seeded by `seed` (cg.hpp:1517-1531).
float ref_hero(uint64_t seed, float* out_lam) {
  nl::RNG rng(seed);
  coefficientλ<Nλ> s(0.f);
  sample::info<heroλ> si;
  sample::spectrum(s, si, rng);
  hero_out(si.val, out_lam);
  return si.prob;
}

// coefficientλ::operator()(heroλ) of one of the scene's spectra.
void ref_eval_spectrum(float const* v80, float const* lam, float* out) {
  coefficientλ<Nλ> c(0.f);
  for (uint32_t i = 0; i < Nλ; i++) c.v[i] = v80[i];
  hero_out(c(hero_from(lam)), out);
}

// coefficientλ::addHeroλ (cg.hpp:306-320) into a zero spectrum.
void ref_add_hero(float const* lam, float const* s, float* out80) {
  coefficientλ<Nλ> c(0.f);
  c.addHeroλ(hero_from(lam), hero_from(s));
  for (uint32_t i = 0; i < Nλ; i++) out80[i] = c.v[i];
}

// coefλ2linRGB (cg.hpp:340-341)
void ref_coef_to_linrgb(float const* v80, float* out3) {
  coefficientλ<Nλ> c(0.f);
  for (uint32_t i = 0; i < Nλ; i++) c.v[i] = v80[i];
  linRGB const x = coefλ2linRGB(c);
  out3[0] = x.c[0];
  out3[1] = x.c[1];
  out3[2] = x.c[2];
}

// BxDFcosθ (cg.hpp:1088-1102) for material `mat` of the loaded scene.
void ref_bxdf(void* h, uint32_t mat, float const* lam, float const* i,
              float const* o, float const* n, int front, float* out) {
  auto* r = static_cast<ref_scene*>(h);
  hero_out(BxDFcosθ(hero_from(lam), r->sc.materials[mat], v3(i), v3(o),
                    v3(n), front != 0),
           out);
}

// sample::materiali (cg.hpp:1953-1968) with an RNG seeded by `seed`.
int ref_sample_material(void* h, float const* lam, ref_hitinfo const* hi,
                        float const* o, uint64_t seed, float p,
                        float* out_prob, float* out_dir, float* out_mult) {
  auto* r = static_cast<ref_scene*>(h);
  nl::RNG rng(seed);
  hitinfo const hinfo = to_hinfo(*hi);
  sample::info<ℝ3, heroλ> si;
  si.prob = 0.f;
  si.val = ℝ3{0.f, 0.f, 0.f};
  si.mult = heroλ(0.f);
  bool const ok = sample::materiali(hero_from(lam), &r->sc.materials[hinfo.mat],
                                    hinfo, v3(o), si, rng, p);
  *out_prob = si.prob;
  put3(si.val, out_dir);
  hero_out(si.mult, out_mult);
  return ok ? 1 : 0;
}

// sample::probForMateriali (cg.hpp:1971-1985), argument order as the
// reference's call site uses it (src/renderer.cpp:136-137).
float ref_prob_for_material(void* h, float l, ref_hitinfo const* hi,
                            float const* i, float const* o, float p) {
  auto* r = static_cast<ref_scene*>(h);
  hitinfo const hinfo = to_hinfo(*hi);
  return sample::probForMateriali(l, &r->sc.materials[hinfo.mat], hinfo, v3(i),
                                  v3(o), p);
}

// sample::light (cg.hpp:1717-1732) for light `light` (includes the shadow
// ray) with an RNG seeded by `seed`.
void ref_sample_light(void* h, uint32_t light, float const* lam,
                      ref_hitinfo const* hi, uint64_t seed, float* out_prob,
                      float* out_dir, float* out_mult) {
  auto* r = static_cast<ref_scene*>(h);
  nl::RNG rng(seed);
  hitinfo const hinfo = to_hinfo(*hi);
  sample::info<ℝ3, heroλ> si;
  si.prob = 0.f;
  si.val = ℝ3{0.f, 0.f, 0.f};
  si.mult = heroλ(0.f);
  sample::light(hero_from(lam), &r->sc.lights[light], hinfo, r->sc, si, rng);
  *out_prob = si.prob;
  put3(si.val, out_dir);
  hero_out(si.mult, out_mult);
}

// sample::probForLight (cg.hpp:1735-1747)
float ref_prob_for_light(void* h, uint32_t light, float const* ray6) {
  auto* r = static_cast<ref_scene*>(h);
  return sample::probForLight(&r->sc.lights[light],
                              ray(v3(ray6), v3(ray6 + 3)));
}

// Renderer::toneMap (src/renderer.cpp:149-176) and rendering::rgb24
// (include/renderer.hpp:20-29).
void ref_tonemap(float const* rgb, uint64_t w, uint64_t h, float y_mid,
                 float* out_tm, uint8_t* out24) {
  rendering in;
  in.img.init(w, h);
  for (uint64_t i = 0; i < w * h; i++)
    in.img.data[i] = linRGB(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
  rendering tm;
  Renderer rd;
  rd.toneMap(in, tm, y_mid);
  for (uint64_t i = 0; i < w * h; i++)
    for (int c = 0; c < 3; c++) out_tm[3 * i + c] = tm.img.data[i].c[c];
  std::vector<rgb24> const b = tm.rgb24();
  for (uint64_t i = 0; i < w * h; i++)
    for (int c = 0; c < 3; c++) out24[3 * i + c] = b[i].c[c];
}

int ref_max_threads() { return omp_get_max_threads(); }

}  // extern "C"
