// lgpu_adjoint.cuh — path-replay backpropagation of the image loss to the
// material parameters (the reference has no derivative code; this is the
// adjoint of Renderer::tracePath, src/renderer.cpp:64-146).
//
// A path's radiance per hero wavelength is
//     L = Σ_v β_v (E_v + N_v),   β_{v+1} = β_v f_v / q_v,
// with E_v the emission found at vertex v, N_v its light sample (the BSDF
// value f(light dir) times the light's weighted radiance, if the shadow ray
// is unoccluded) and f_v / q_v the material sample's BSDF value over its
// (MIS-weighted) density.  For a parameter π of the material at vertex v,
// with sampling decisions and MIS weights held fixed,
//     dL/dπ = β_v ∂N_v/∂π + L_after_v ∂ln f_v/∂π,
// where L_after_v = Σ_{w>v} β_w (E_w + N_w) is the radiance the path
// gathers after v.  Two passes per chunk of work items:
//   primal  the wavefront render, which also stores every path's L and a bit
//           per vertex telling whether its shadow ray reached the light;
//   replay  the same paths again from their random streams (no shadow rays:
//           visibility comes from the bits), starting from L and subtracting
//           each vertex's contribution to get L_after_v, accumulating
//           dL/dπ · dLoss/dL into the gradients.
// Parameters: the bins of Lambertian albedo spectra and of thin-film IOR
// spectra, thin-film thickness, and the exponent α of Blinn and thin-film
// lobes.
#pragma once

#include "lgpu_render.cuh"

namespace lgpu {

// ---- forward-mode derivatives of thinfilm::BRDFcosθ ------------------------------

// value and derivatives along two directions (film IOR n1, thickness d)
struct Dual2 {
  float v, a, b;
};
__device__ __forceinline__ Dual2 dc(float x) { return Dual2{x, 0.f, 0.f}; }
__device__ __forceinline__ Dual2 operator+(Dual2 x, Dual2 y) { return Dual2{x.v + y.v, x.a + y.a, x.b + y.b}; }
__device__ __forceinline__ Dual2 operator-(Dual2 x, Dual2 y) { return Dual2{x.v - y.v, x.a - y.a, x.b - y.b}; }
__device__ __forceinline__ Dual2 operator*(Dual2 x, Dual2 y) {
  return Dual2{x.v * y.v, x.a * y.v + x.v * y.a, x.b * y.v + x.v * y.b};
}
__device__ __forceinline__ Dual2 operator/(Dual2 x, Dual2 y) {
  float const q = x.v / y.v;
  return Dual2{q, (x.a - q * y.a) / y.v, (x.b - q * y.b) / y.v};
}
__device__ __forceinline__ Dual2 dsqrt(Dual2 x) {
  float const r = sqrtf(x.v);
  float const h = r > 0.f ? 0.5f / r : 0.f;
  return Dual2{r, x.a * h, x.b * h};
}
__device__ __forceinline__ Dual2 dcos(Dual2 x) {
  float s, c;
  sincosf(x.v, &s, &c);
  return Dual2{c, -s * x.a, -s * x.b};
}

// thinfilm_k (lgpu_path.cuh, cg.hpp:1001-1051) with its value's derivatives
// with respect to the film IOR n1 (.a) and the thickness d (.b)
__device__ __forceinline__ Dual2 thinfilm_dual(float n1v, float n2v, float dv, float alpha, float l, float cos_i,
                                               float pow5, float pow_hn) {
  Dual2 const n1{n1v, 1.f, 0.f}, n2 = dc(n2v), d{dv, 0.f, 1.f};
  Dual2 const one = dc(1.f);
  Dual2 const n01 = one / n1;
  Dual2 const cos_l = dsqrt(one - n01 * n01) * dc(1.f - cos_i * cos_i);
  Dual2 const cos_d = dcos(dc(4.f * kPi) * n1 * d * cos_l / dc(l));
  Dual2 const a01 = one - n1, b01 = one + n1;
  Dual2 const R0_01 = a01 * a01 / (b01 * b01);
  Dual2 const a12 = n1 - n2, b12 = n1 + n2;
  Dual2 const R0_12 = a12 * a12 / (b12 * b12);
  Dual2 const R01 = R0_01 + (one - R0_01) * dc(pow5);
  Dual2 const R12 = R0_12 + (one - R0_12) * dc(pow5);
  Dual2 const Ravg = dc(2.f) * dsqrt(R01 * R12);
  Dual2 const Rt = (R01 + R12 + Ravg * cos_d) / (one + R01 * R12 + Ravg * cos_d);
  return dc((alpha + 2.f) * 0.125f * kInvPi * pow_hn) * Rt;
}

// ---- accumulation ---------------------------------------------------------------

// v * d spec_at(S, s, x) / d bins of spectrum s (the lerp of spec_at)
__device__ __forceinline__ void spec_grad(const DevScene& S, float* g_spec, int32_t s, float x, float v) {
  if (v == 0.f || !isfinite(v)) return;
  float* g = g_spec + size_t(s) * S.n_bins;
  uint32_t const n = S.n_bins;
  if (x < 0.f) {
    atomicAdd(g, v);
    return;
  }
  if (x >= 1e29f) {
    atomicAdd(g + n - 1, v);
    return;
  }
  uint32_t const i = min(uint32_t(x), n - 2);
  float const t = x - float(i);
  atomicAdd(g + i, v * (1.f - t));
  atomicAdd(g + i + 1, v * t);
}

// d ln(pow(hn, α) (α+2)) / dα, or 0 where the lobe value is 0
__device__ __forceinline__ float dlog_lobe_dalpha(float alpha, float c, float lnhn) {
  return c > 0.f ? 1.f / (alpha + 2.f) + lnhn : 0.f;
}

// v * d BxDFcosθ(light dir) / dπ for the NEE term (bsdf_k's cases)
__device__ __forceinline__ void grad_bsdf(const DevScene& S, const DevMaterial& m, uint32_t mat,
                                          const BsdfScalars& r, float x, float l, bool front, float v,
                                          const AdjointArgs& g, float& g_d, float& g_alpha) {
  switch (r.kind) {
    case 1:
      spec_grad(S, g.g_spec, m.spectrum[0], x, v * kInvPi * r.a);
      break;
    case 2:
    case 3: {
      float const ior = spec_at(S, m.spectrum[4], x);
      float const eta = front ? 1.f / ior : ior;
      float const F0 = schlick_F0(eta);
      float const F = F0 + (1.f - F0) * r.b;
      float const gl = (m.alpha + 2.f) * 0.125f * kInvPi * r.c;
      float const spec = r.kind == 2 ? (spec_at(S, m.spectrum[1], x) + F * spec_at(S, m.spectrum[2], x)) * gl
                                     : spec_at(S, m.spectrum[2], x) * (1.f - F) * gl;
      g_alpha += v * spec * dlog_lobe_dalpha(m.alpha, r.c, r.lnhn);
      break;
    }
    case 4: {
      Dual2 const f = thinfilm_dual(spec_at(S, m.spectrum[0], x), spec_at(S, m.spectrum[1], x), m.d, m.alpha, l,
                                    r.a, r.b, r.c);
      spec_grad(S, g.g_spec, m.spectrum[0], x, v * f.a);
      g_d += v * f.b;
      g_alpha += v * f.v * dlog_lobe_dalpha(m.alpha, r.c, r.lnhn);
      break;
    }
  }
  (void)mat;
}

// u * d ln f / dπ for the material sample's BSDF value f = mat_mult_k
// (u = dLoss/dL * L_after at this wavelength)
__device__ __forceinline__ void grad_mult(const DevScene& S, const DevMaterial& m, const MatSample& ms, float x,
                                          float l, float f, float u, const AdjointArgs& g, float& g_d,
                                          float& g_alpha) {
  if (f == 0.f || u == 0.f) return;
  switch (ms.lobe) {
    case 1:
      if (m.type == LGPU_MAT_LAMBERTIAN) {
        float const alb = spec_at(S, m.spectrum[0], x);
        if (alb != 0.f) spec_grad(S, g.g_spec, m.spectrum[0], x, u / alb);
      }
      break;
    case 2:
    case 3:
      g_alpha += u * dlog_lobe_dalpha(m.alpha, ms.c, ms.lnhn);
      break;
    case 4: {
      Dual2 const t = thinfilm_dual(spec_at(S, m.spectrum[0], x), spec_at(S, m.spectrum[1], x), m.d, m.alpha, l,
                                    ms.a, ms.b, ms.c);
      if (t.v != 0.f) {
        spec_grad(S, g.g_spec, m.spectrum[0], x, u * t.a / t.v);
        g_d += u * t.b / t.v;
      }
      g_alpha += u * dlog_lobe_dalpha(m.alpha, ms.c, ms.lnhn);
      break;
    }
  }
}

namespace {

// Replay: the chunk's paths restart from their random streams with the
// radiance the primal pass recorded and their dLoss/dL weights:
//     dLoss/dL_k = Σ_c dLoss/dRGB_c (M_XYZ→RGB · w_XYZ(λ_k))_c Δ / (spp K p(λ))
// with w_XYZ(λ) the XYZ of addHeroλ(λ, 1) (cg.hpp:306-320, 283-288).
template <int K>
__global__ void __launch_bounds__(256) wf_replay_generate(OneJob jobs, WaveState w, AdjointArgs g) {
  uint32_t const n_new = w.ctl[kCtlNew], first = w.ctl[kCtlFirst], pos = w.ctl[kCtlPos];
  uint32_t const cap = w.cap;
  const DevScene& S = jobs.S;
  const RenderArgs& a = jobs.a;
  PathBuf const& in = w.in;
  float const omega = S.lambda_sup - S.lambda_inf;
  float const step = omega / float(K);
  const lgpu_camera& C = S.cam;
  uint32_t const W = uint32_t(C.width), H = uint32_t(C.height);
  float const scale = S.lambda_delta / (float(a.spp) * float(K)) * omega;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_new; k += gridDim.x * blockDim.x) {
    uint32_t const q = first + k;
    uint64_t const gq = w.c0 + q;
    uint32_t const sample = uint32_t(gq / jobs.npix);
    uint32_t const pix = uint32_t(gq - uint64_t(sample) * jobs.npix);
    uint32_t const p = pos + k;
    uint32_t const i = pix / W, j = pix - i * W;
    uint64_t rng = lgpu_path_state(a.seed, (uint64_t(a.stream_tag) << 32) | pix, uint64_t(a.spp_offset) + sample);
    float const u = float(j) + lgpu_flt(&rng);
    float const v = float(i) + lgpu_flt(&rng);
    f3 const Fx = f3{C.base_x[0], C.base_x[1], C.base_x[2]};
    f3 const Fy = f3{C.base_y[0], C.base_y[1], C.base_y[2]};
    f3 const Fz = f3{C.base_z[0], C.base_z[1], C.base_z[2]};
    f3 const P = f3{C.pos[0], C.pos[1], C.pos[2]};
    float const cu = -0.5f * C.w + C.delta * u;
    float const cv = -0.5f * C.h + C.delta * v;
    f3 const wij = f3{P.x + Fx.x * cu + Fy.x * cv - C.D * Fz.x, P.y + Fx.y * cu + Fy.y * cv - C.D * Fz.y,
                      P.z + Fx.z * cu + Fy.z * cv - C.D * Fz.z};
    float const la = lgpu_flt(&rng) - 0.5f;
    float const lb = lgpu_flt(&rng) - 0.5f;
    float const dd = 2.f * C.dof;
    f3 const wkl = f3{P.x + dd * (Fx.x * la + Fy.x * lb), P.y + dd * (Fx.y * la + Fy.y * lb),
                      P.z + dd * (Fx.z * la + Fy.z * lb)};
    f3 const dir = fnorm(f3{wij.x - wkl.x, wij.y - wkl.y, wij.z - wkl.z});
    float const hero = S.lambda_inf + omega * lgpu_flt(&rng);
    in.ray[0 * cap + p] = wkl.x;
    in.ray[1 * cap + p] = wkl.y;
    in.ray[2 * cap + p] = wkl.z;
    in.ray[3 * cap + p] = dir.x;
    in.ray[4 * cap + p] = dir.y;
    in.ray[5 * cap + p] = dir.z;
    in.rng[p] = rng;
    in.hero[p] = hero;
    in.depth[p] = 0;
    in.item[p] = q;
    const float* dI = g.dimg + (size_t(H - i - 1) * W + j) * 3;
    float const dR = dI[0], dG = dI[1], dB = dI[2];
    // dLoss/dXYZ through the XYZ -> linear RGB matrix of finalize
    float const dX = 3.2404542f * dR - 0.9692660f * dG + 0.0556434f * dB;
    float const dY = -1.5371385f * dR + 1.8760108f * dG - 0.2040259f * dB;
    float const dZ = -0.4985314f * dR + 0.0415560f * dG + 1.0572252f * dB;
#pragma unroll
    for (int kk = 0; kk < K; kk++) {
      float X = 0.f, Y = 0.f, Z = 0.f;
      splat_xyz(S, hero_lambda(S, hero, step, kk), 1.f, X, Y, Z);
      in.beta[kk * cap + p] = 1.f;
      in.acc[kk * cap + p] = w.ltot[size_t(q) * K + kk];
      in.gw[kk * cap + p] = (dX * X + dY * Y + dZ * Z) * scale;
    }
  }
}

// One vertex of the replay: the same random decisions as wf_shade, the
// visibility recorded by the primal pass, gradients accumulated.
template <int K>
// 10 blocks of 128 per SM: like the forward shading, latency-bound, so more
// warps beat fewer spills (5 blocks at 89 registers made the adjoint 5 %
// slower).
__global__ void __launch_bounds__(128, 10) wf_shade_adjoint(OneJob jobs, WaveState w, AdjointArgs g) {
  uint32_t const n = *w.n_in;
  uint32_t const cap = w.cap;
  const DevScene& S = jobs.S;
  const RenderArgs& a = jobs.a;
  PathBuf const& in = w.in;
  PathBuf const& out = w.out;
  float const omega = S.lambda_sup - S.lambda_inf;
  float const step = omega / float(K);
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t const i = material_order(jobs, w, base, n);
    bool const live = i < n;
    bool cont = false, scatter = false, visible = false;
    f3 np = f3{0.f, 0.f, 0.f}, nd = f3{0.f, 0.f, 1.f};
    float lis_scale = 0.f, m_scale = 0.f, hero = 0.f;
    // d ln w_L / dα and d ln w_mat / dα of the MIS weights (below)
    float dlw_L = 0.f, dlw_mat = 0.f;
    uint64_t rng = 0;
    uint32_t mat = 0, light = 0, depth = 0;
    bool front = true;
    MatSample ms;
    ms.ok = false;
    BsdfScalars bl{};
    if (live) {
      hero = in.hero[i];
      depth = in.depth[i];
      HitRec h;
      h.obj = __float_as_uint(w.hit[cap + i]);
      if (h.obj != UINT32_MAX) {
        h.z = w.hit[i];
        h.face = __float_as_uint(w.hit[2 * cap + i]);
        h.b0 = w.hit[3 * cap + i];
        h.b1 = w.hit[4 * cap + i];
        h.b2 = w.hit[5 * cap + i];
        h.pl = f3{w.hit[6 * cap + i], w.hit[7 * cap + i], w.hit[8 * cap + i]};
        Ray const r = load_ray(in.ray, cap, i);
        HitInfo const H = finalize_hit(S, r, h);
        f3 const un = fnorm(r.u);
        f3 const o = f3{-un.x, -un.y, -un.z};
        f3 const nn = H.front ? H.F.z : neg3(H.F.z);
        mat = H.mat;
        front = H.front;
        const DevMaterial& m = S.mats[mat];
        // an emitter ends the path; its radiance is not a parameter
        if (m.type != LGPU_MAT_EMITTER && m.type != LGPU_MAT_DIREMITTER && depth <= a.max_scatter) {
          scatter = true;
          rng = in.rng[i];
          light = uint32_t(lgpu_u64(&rng) % uint64_t(S.n_lights));
          float const prob_l = 1.f / float(S.n_lights);
          const lgpu_light& L = S.lights[light];
          float stmax = 0.f;
          uint32_t sskip = UINT32_MAX;
          LightSample ls = sample_light_unoccluded(S, L, H, rng, stmax, sskip);
          float const x0 = lam_coord(S, hero);
          bl = bsdf_scalars(S, m, x0, ls.dir, o, nn, H.front);
          ms = sample_material(S, m, x0, H, o, a.sample_p, rng);
          float w_L = 1.f, w_mat = 0.f;
          if (ms.ok) {
            float const p_L_mati = prob_for_light(S, L, H.p, ms.dir) * prob_l;
            float dlp_Li = 0.f;
            float const p_mat_Li = prob_for_material(S, m, x0, H, ls.dir, o, a.sample_p, &dlp_Li);
            float const p_L_i = ls.prob * prob_l;
            w_L = p_L_i * p_L_i / (p_L_i * p_L_i + p_mat_Li * p_mat_Li);
            w_mat = ms.prob * ms.prob / (ms.prob * ms.prob + p_L_mati * p_L_mati);
            // The power-heuristic weights depend on α through the material
            // pdf (at the light sample's direction for w_L, at the material
            // sample's for w_mat).  In a proper MIS their derivatives would
            // cancel in expectation; here they do not, because the
            // reference applies w_L only when a material sample exists
            // (src/renderer.cpp:120) and w_mat to the whole recursive
            // radiance (src/renderer.cpp:145), so the gradient of its
            // expected image carries them:
            //   d ln w_L / dα   = -2 (1 - w_L) d ln p_mat(ω_L) / dα
            //   d ln w_mat / dα =  2 (1 - w_mat) d ln p_mat(ω_mat) / dα
            // (the sample's own 1/pdf needs no term: its α-derivative equals
            // the score of the density the direction was drawn from).
            dlw_L = -2.f * (1.f - w_L) * dlp_Li;
            dlw_mat = 2.f * (1.f - w_mat) * ms.dlnprob;
          }
          lis_scale = ls.scale / (ls.prob * prob_l) * w_L;
          m_scale = ms.ok ? w_mat / ms.prob : 0.f;
          bool const needs_test = stmax >= 0.f;
          visible = !needs_test || ((w.vis[in.item[i]] >> depth) & 1ull);
          cont = ms.ok;
          if (cont) {
            np = H.p;
            nd = ms.dir;
          }
        }
      }
    }
    uint32_t const o_pos = warp_append(w.n_out, cont);
    if (!scatter) continue;
    const DevMaterial& m = S.mats[mat];
    const lgpu_light& L = S.lights[light];
    float g_d = 0.f, g_alpha = 0.f;
    for (int k = 0; k < K; k++) {
      float const l = hero_lambda(S, hero, step, k);
      float const x = lam_coord(S, l);
      float const b = in.beta[k * cap + i];
      float const gw = in.gw[k * cap + i];
      float rem = in.acc[k * cap + i];
      if (visible && lis_scale != 0.f) {
        float const coef = bsdf_k(S, m, bl, x, l, front);
        float const rad = spec_at(S, L.spectrum, x);
        grad_bsdf(S, m, mat, bl, x, l, front, gw * b * rad * lis_scale, g, g_d, g_alpha);
        float const nee = b * (rad * coef * lis_scale);
        g_alpha += gw * nee * dlw_L;
        rem -= nee;
      }
      if (cont) {
        float const f = mat_mult_k(S, m, ms, x, l, front);
        grad_mult(S, m, ms, x, l, f, gw * rem, g, g_d, g_alpha);
        g_alpha += gw * rem * dlw_mat;
        out.beta[k * cap + o_pos] = b * (f * m_scale);
        out.acc[k * cap + o_pos] = rem;
        out.gw[k * cap + o_pos] = gw;
      }
    }
    if (g_d != 0.f && isfinite(g_d)) atomicAdd(g.g_mat + 4 * size_t(mat), g_d);
    if (g_alpha != 0.f && isfinite(g_alpha)) atomicAdd(g.g_mat + 4 * size_t(mat) + 1, g_alpha);
    if (cont) {
      out.ray[0 * cap + o_pos] = np.x;
      out.ray[1 * cap + o_pos] = np.y;
      out.ray[2 * cap + o_pos] = np.z;
      out.ray[3 * cap + o_pos] = nd.x;
      out.ray[4 * cap + o_pos] = nd.y;
      out.ray[5 * cap + o_pos] = nd.z;
      out.rng[o_pos] = rng;
      out.hero[o_pos] = hero;
      out.depth[o_pos] = depth + 1;
      out.item[o_pos] = in.item[i];
    }
  }
}

}  // namespace

// The replay pass over work items [c0, c0 + total).
template <int K>
cudaError_t replay_chunk(const OneJob& jobs, WaveState& w, uint64_t c0, uint32_t total, bool linear,
                         const AdjointArgs& g, DevCounters* d_cnt, cudaStream_t st, WaveLaunch* run) {
  static uint32_t gen_per_sm = 0;
  if (!gen_per_sm) gen_per_sm = blocks_per_sm(wf_replay_generate<K>, 256, 0);
  WaveGrids const gr = wave_grids<K, OneJob>(run->cfg);
  uint32_t const sms = wave_occupancy<K, OneJob>().sms;
  DevCounters* const c_closest = run->on ? d_cnt + 1 : d_cnt;
  w.c0 = c0;
  wf_stream_init<<<1, 32, 0, st>>>(w);
  run->total++;
  return run_iterations(w, total, st, run, [&](const WaveState& wi) {
    wf_plan<<<1, 1, 0, st>>>(wi, total);
    wf_replay_generate<K><<<sms * gen_per_sm, 256, 0, st>>>(jobs, wi, g);
    run->begin(0, st);
    launch_closest<K>(jobs, wi, gr, linear, c_closest, st);
    run->end(0, st);
    run->begin(2, st);
    // one block per queue chunk (see wave_chunk)
    wf_shade_adjoint<K><<<(wi.cap + 127) / 128, 128, 0, st>>>(jobs, wi, g);
    run->end(2, st);
    // plan, generate, trace (+ fallback), shade
    run->total += linear ? 4 : 5;
  });
}

// Primal render (image into d_img when not null) and gradients, chunk by
// chunk: the primal pass records, the replay pass differentiates.
template <int K>
cudaError_t launch_adjoint_k(const DevScene& S, const RenderArgs& a, WaveState* wave, uint64_t chunk_items,
                             float* d_img, const AdjointArgs& g, DevCounters* d_cnt, cudaStream_t st,
                             WaveLaunch* run) {
  OneJob const jobs{S, a, wave->npix, d_img};
  WaveState w = *wave;
  bool const linear = (a.flags & LGPU_FLAG_REFERENCE_ORDER) || S.n_objects <= 4;
  uint64_t const n_items = uint64_t(wave->npix) * a.spp;
  cudaError_t e = cudaMemsetAsync(w.film, 0, sizeof(float) * 3 * size_t(w.npix), st);
  for (uint64_t c0 = 0; c0 < n_items && e == cudaSuccess; c0 += chunk_items) {
    uint32_t const total = uint32_t(n_items - c0 < chunk_items ? n_items - c0 : chunk_items);
    e = wave_chunk<K>(jobs, w, c0, total, linear, d_cnt, st, run);
    if (e == cudaSuccess) e = replay_chunk<K>(jobs, w, c0, total, linear, g, d_cnt, st, run);
  }
  if (e == cudaSuccess && d_img) e = finalize_film<K>(jobs, w, st, run);
  return e;
}

}  // namespace lgpu
