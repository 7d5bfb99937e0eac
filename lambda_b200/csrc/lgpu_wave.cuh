// lgpu_wave.cuh — wavefront path tracing.
//
// A wave is a set of paths (n_samples samples of every pixel) processed one
// bounce at a time by short kernels over compacted queues:
//
//   wf_generate   camera ray + hero wavelengths of every path of the wave
//   wf_trace      closest hit of every active path          (queue q_in)
//   wf_shade<K>   emitters, light sample -> shadow ray, material sample ->
//                 next ray, throughput update                 (q_in -> q_out,
//                 shadow queue)
//   wf_shadow<K>  any-hit test of the shadow rays; adds their radiance
//   wf_splat<K>   adds every path's radiance to its pixel's XYZ film
//   wf_finalize   film -> linear RGB in the reference's layout
//
// Each path draws its random numbers from its own counter-based stream in
// the same order as Renderer::tracePath (src/renderer.cpp:64-146), so a
// path's result does not depend on which kernel or slot processes it.
// Paths are appended to the output queues with one atomic per warp
// (ballot + popc).  The per-path state is SoA so a warp's accesses to one
// field are coalesced.  Spectral state (throughput and radiance per hero
// wavelength) lives in memory and is streamed one wavelength at a time, so
// the shading kernel keeps no spectral arrays in registers.
#pragma once

#include "lgpu_counters.cuh"
#include "lgpu_path.cuh"
#include "lgpu_traverse.cuh"

namespace lgpu {

__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool pred) {
  unsigned const mask = __activemask();
  unsigned const b = __ballot_sync(mask, pred);
  int const lane = threadIdx.x & 31;
  int const leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader && b) base = atomicAdd(counter, __popc(b));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(b & ((1u << lane) - 1u));
}

// The non-template kernels get internal linkage: every translation unit
// that instantiates the renderer carries its own copy.
namespace {

// ---- generate -------------------------------------------------------------------

__global__ void __launch_bounds__(256) wf_generate(DevScene S, RenderArgs a, WaveState w, uint32_t k_hero,
                                                   uint32_t sample_base, DevCounters* cnt) {
  uint32_t const n = w.npix * w.n_samples;
  uint32_t paths = 0;
  float const omega = S.lambda_sup - S.lambda_inf;
  const lgpu_camera& C = S.cam;
  uint32_t const W = uint32_t(C.width);
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    uint32_t const s_local = p / w.npix;
    uint32_t const pix = p - s_local * w.npix;
    uint32_t const i = pix / W, j = pix - i * W;
    uint64_t rng = lgpu_path_state(a.seed, (uint64_t(a.stream_tag) << 32) | pix,
                                   uint64_t(a.spp_offset) + sample_base + s_local);
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
    uint32_t const cap = w.cap;
    w.ray[0 * cap + p] = wkl.x;
    w.ray[1 * cap + p] = wkl.y;
    w.ray[2 * cap + p] = wkl.z;
    w.ray[3 * cap + p] = dir.x;
    w.ray[4 * cap + p] = dir.y;
    w.ray[5 * cap + p] = dir.z;
    w.rng[p] = rng;
    w.hero[p] = hero;
    w.depth[p] = 0;
    for (uint32_t k = 0; k < k_hero; k++) {
      w.beta[k * cap + p] = 1.f;
      w.acc[k * cap + p] = 0.f;
    }
    w.q_in[p] = p;
    paths++;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *w.n_in = n;
  TravStats const ts{0u, 0u, 0u, 0u};
  flush_counters(cnt, 0u, paths, ts, 0u);
}

// ---- trace ------------------------------------------------------------------------

__global__ void __launch_bounds__(128) wf_trace(DevScene S, WaveState w, uint32_t flags, DevCounters* cnt) {
  extern __shared__ StackEntry smem_stack[];
  StackEntry lm[kLocalStack];
  StackEntry lstack[kStackCap];
  StackEntry ltstack[kTlasStackCap];
  SplitStack st{smem_stack + threadIdx.x, blockDim.x, lm, 0};
  TravStats ts{0u, 0u, 0u, 0u};
  uint32_t rays = 0;
  bool const ref_order = (flags & LGPU_FLAG_REFERENCE_ORDER) != 0;
  uint32_t const n = *w.n_in;
  uint32_t const cap = w.cap;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t const p = w.q_in[i];
    Ray const r = make_ray(f3{w.ray[p], w.ray[cap + p], w.ray[2 * cap + p]},
                           f3{w.ray[3 * cap + p], w.ray[4 * cap + p], w.ray[5 * cap + p]});
    HitRec h;
    h.z = kFltMax;
    h.obj = UINT32_MAX;
    h.face = UINT32_MAX;
    h.b0 = h.b1 = h.b2 = 0.f;
    h.pl = f3{0.f, 0.f, 0.f};
    scene_trace<false>(S, r, h, UINT32_MAX, ref_order, st, lstack, ltstack, ts);
    rays++;
    float* hp = w.hit;
    hp[0 * cap + p] = h.z;
    hp[1 * cap + p] = __uint_as_float(h.obj);
    hp[2 * cap + p] = __uint_as_float(h.face);
    hp[3 * cap + p] = h.b0;
    hp[4 * cap + p] = h.b1;
    hp[5 * cap + p] = h.b2;
    hp[6 * cap + p] = h.pl.x;
    hp[7 * cap + p] = h.pl.y;
    hp[8 * cap + p] = h.pl.z;
  }
  flush_counters(cnt, rays, 0u, ts, 0u);
}

// ---- streaming scheduler ------------------------------------------------------------

// All slots free, no work handed out, no path in flight.
__global__ void wf_stream_init(WaveState w) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < w.cap; p += gridDim.x * blockDim.x)
    w.free_list[p] = p;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    w.ctl[0] = w.cap;
    w.ctl[1] = 0;
    w.ctl[2] = 0;
    *w.n_in = 0;
  }
}

// Decides how many new paths the next generate starts: as many as there
// are free slots, up to the remaining work items.
__global__ void wf_plan(WaveState w, uint32_t total) {
  uint32_t const n_free = w.ctl[0], next = w.ctl[1];
  uint32_t const left = total - next;
  uint32_t const n_new = n_free < left ? n_free : left;
  w.ctl[3] = n_new;
  w.ctl[4] = next;
  w.ctl[5] = n_free;
  w.ctl[6] = *w.n_in;
  w.ctl[0] = n_free - n_new;
  w.ctl[1] = next + n_new;
  *w.n_in += n_new;
}

// Starts the planned paths: work item q is sample q / npix of pixel
// q % npix (all pixels of one sample before the next sample).
__global__ void __launch_bounds__(256) wf_generate_stream(DevScene S, RenderArgs a, WaveState w,
                                                          uint32_t k_hero, uint32_t sample_base,
                                                          DevCounters* cnt) {
  uint32_t const n_new = w.ctl[3], first = w.ctl[4], top = w.ctl[5], qpos = w.ctl[6];
  uint32_t paths = 0;
  float const omega = S.lambda_sup - S.lambda_inf;
  const lgpu_camera& C = S.cam;
  uint32_t const W = uint32_t(C.width);
  uint32_t const cap = w.cap;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_new; k += gridDim.x * blockDim.x) {
    uint32_t const q = first + k;
    uint32_t const s_local = q / w.npix;
    uint32_t const pix = q - s_local * w.npix;
    uint32_t const p = w.free_list[top - 1 - k];
    uint32_t const i = pix / W, j = pix - i * W;
    uint64_t rng = lgpu_path_state(a.seed, (uint64_t(a.stream_tag) << 32) | pix,
                                   uint64_t(a.spp_offset) + sample_base + s_local);
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
    w.ray[0 * cap + p] = wkl.x;
    w.ray[1 * cap + p] = wkl.y;
    w.ray[2 * cap + p] = wkl.z;
    w.ray[3 * cap + p] = dir.x;
    w.ray[4 * cap + p] = dir.y;
    w.ray[5 * cap + p] = dir.z;
    w.rng[p] = rng;
    w.hero[p] = hero;
    w.depth[p] = 0;
    w.pix[p] = pix;
    w.samp[p] = s_local;
    for (uint32_t kk = 0; kk < k_hero; kk++) {
      w.beta[kk * cap + p] = 1.f;
      w.acc[kk * cap + p] = 0.f;
    }
    w.q_in[qpos + k] = p;
    paths++;
  }
  TravStats const ts{0u, 0u, 0u, 0u};
  flush_counters(cnt, 0u, paths, ts, 0u);
}

// Ended paths: their radiance goes to the (sample, pixel) film entry, their
// slot back to the free list.
template <int K>
__global__ void __launch_bounds__(256) wf_finish(DevScene S, WaveState w, DevCounters* cnt) {
  uint32_t const n = w.ctl[2];
  float const omega = S.lambda_sup - S.lambda_inf;
  float const step = omega / float(K);
  float const prob_l = 1.f / omega;
  uint32_t nonfinite = 0;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t const i = base + threadIdx.x;
    bool const live = i < n;
    uint32_t p = 0;
    if (live) {
      p = w.fin_list[i];
      float const hero = w.hero[p];
      float sx = 0.f, sy = 0.f, sz = 0.f;
      bool finite = true;
      for (int k = 0; k < K; k++) {
        float const val = w.acc[k * w.cap + p] / prob_l;
        finite = finite && isfinite(val);
        splat_xyz(S, hero_lambda(S, hero, step, k), val, sx, sy, sz);
      }
      nonfinite += finite ? 0u : 1u;
      size_t const o = 3 * (size_t(w.samp[p]) * w.npix + w.pix[p]);
      w.sbuf[o] = sx;
      w.sbuf[o + 1] = sy;
      w.sbuf[o + 2] = sz;
    }
    uint32_t const slot = warp_append(&w.ctl[0], live);
    if (live) w.free_list[slot] = p;
  }
  TravStats const ts{0u, 0u, 0u, 0u};
  flush_counters(cnt, 0u, 0u, ts, nonfinite);
}

// Film: per pixel, the (sample, pixel) entries summed in sample order.
__global__ void __launch_bounds__(256) wf_reduce(WaveState w, uint32_t n_samples) {
  for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < w.npix; pix += gridDim.x * blockDim.x) {
    float X = w.film[3 * pix], Y = w.film[3 * pix + 1], Z = w.film[3 * pix + 2];
    for (uint32_t s = 0; s < n_samples; s++) {
      size_t const o = 3 * (size_t(s) * w.npix + pix);
      X += w.sbuf[o];
      Y += w.sbuf[o + 1];
      Z += w.sbuf[o + 2];
    }
    w.film[3 * pix] = X;
    w.film[3 * pix + 1] = Y;
    w.film[3 * pix + 2] = Z;
  }
}

// Persistent instance-BVH traversal of the extension rays (ANY = false,
// queue q_in, hit records out) or the shadow rays (ANY = true, shadow
// queue, unoccluded contributions added to the path radiance).  A lane that
// finishes its ray takes the next one; idle lanes are refilled together with
// one atomic per warp once kRefill of them are waiting.
constexpr int kRefill = 8;

__device__ __forceinline__ void store_hit(const WaveState& w, uint32_t p, const HitRec& h) {
  uint32_t const cap = w.cap;
  float* hp = w.hit;
  hp[0 * cap + p] = h.z;
  hp[1 * cap + p] = __uint_as_float(h.obj);
  hp[2 * cap + p] = __uint_as_float(h.face);
  hp[3 * cap + p] = h.b0;
  hp[4 * cap + p] = h.b1;
  hp[5 * cap + p] = h.b2;
  hp[6 * cap + p] = h.pl.x;
  hp[7 * cap + p] = h.pl.y;
  hp[8 * cap + p] = h.pl.z;
}

template <bool ANY, int K>
__global__ void __launch_bounds__(128, 6) wf_trace_persistent(DevScene S, WaveState w, DevCounters* cnt) {
  extern __shared__ StackEntry smem_stack[];
  StackEntry lm[kLocalStack];
  SplitStack st{smem_stack + threadIdx.x, blockDim.x, lm, 0};
  TravStats ts{0u, 0u, 0u, 0u};
  uint32_t rays = 0;
  uint32_t const n = ANY ? *w.n_shadow : *w.n_in;
  uint32_t* fetch = ANY ? w.fetch + 1 : w.fetch;
  uint32_t const cap = w.cap;
  unsigned const FULL = 0xFFFFFFFFu;
  int const lane = threadIdx.x & 31;
  TraceState t;
  bool active = false, exhausted = false;
  uint32_t idx = 0, wobj = 0;
  int phase = 1;
  while (true) {
    unsigned const idle = __ballot_sync(FULL, !active);
    if (!exhausted && (__popc(idle) >= kRefill || idle == FULL)) {
      int const leader = __ffs(idle) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(fetch, uint32_t(__popc(idle)));
      base = __shfl_sync(FULL, base, leader);
      if (base + uint32_t(__popc(idle)) >= n) exhausted = true;
      if (!active) {
        uint32_t const my = base + uint32_t(__popc(idle & ((1u << lane) - 1u)));
        if (my < n) {
          idx = my;
          if (ANY) {
            t.w = make_ray(f3{w.sray[my], w.sray[cap + my], w.sray[2 * cap + my]},
                           f3{w.sray[3 * cap + my], w.sray[4 * cap + my], w.sray[5 * cap + my]});
            t.h.z = w.sray[6 * cap + my];
            t.skip = __float_as_uint(w.sray[7 * cap + my]);
          } else {
            uint32_t const p = w.q_in[my];
            idx = p;
            t.w = make_ray(f3{w.ray[p], w.ray[cap + p], w.ray[2 * cap + p]},
                           f3{w.ray[3 * cap + p], w.ray[4 * cap + p], w.ray[5 * cap + p]});
            t.h.z = kFltMax;
            t.skip = UINT32_MAX;
          }
          t.h.obj = UINT32_MAX;
          t.h.face = UINT32_MAX;
          t.h.b0 = t.h.b1 = t.h.b2 = 0.f;
          t.h.pl = f3{0.f, 0.f, 0.f};
          t.any = ANY;
          t.ilimit = UINT32_MAX;
          phase = 1;
          trace_begin(S, t, st);
          active = true;
          rays++;
        }
      }
    }
    if (__all_sync(FULL, !active)) {
      if (exhausted) break;
      continue;
    }
    if (active && trace_step<ANY>(S, t, st, ts)) {
      active = false;
      if (ANY) {
        if (!t.hit_any) {
          uint32_t const p = w.s_path[idx];
          for (int k = 0; k < K; k++) w.acc[k * cap + p] += w.s_contrib[k * cap + p];
        }
        continue;
      }
      uint32_t const p = idx;
      if (phase == 2) {
        // an object below W's index is hit before the ray leaves W's bounds:
        // the reference skips W, so its answer is the closest hit without W
        if (t.hit_any) {
          t.w = make_ray(f3{w.ray[p], w.ray[cap + p], w.ray[2 * cap + p]},
                         f3{w.ray[3 * cap + p], w.ray[4 * cap + p], w.ray[5 * cap + p]});
          t.h.z = kFltMax;
          t.h.obj = UINT32_MAX;
          t.h.face = UINT32_MAX;
          t.any = false;
          t.skip = wobj;
          t.ilimit = UINT32_MAX;
          phase = 3;
          trace_begin(S, t, st);
          active = true;
        }
        continue;
      }
      if (phase == 1 && t.hit_any && t.h.inside && t.h.exit > t.h.z) {
        // The winner W is a mesh whose bounds contain the ray origin and
        // which the ray leaves after the hit; the reference skips W if an
        // object tested before it (lower index) was hit before that exit
        // (cg.hpp:1393, 1414).  With W the only such mesh, one any-hit query
        // over the lower-index objects up to the exit decides it; otherwise
        // the ray is re-traced with the linear object loop.
        if (t.n_inside != 1) {
          w.fb_queue[atomicAdd(w.n_fb, 1u)] = p;
          continue;
        }
        store_hit(w, p, t.h);
        wobj = t.h.obj;
        float const ex = t.h.exit;
        t.h.z = prev_float(ex);
        t.h.obj = UINT32_MAX;
        t.any = true;
        t.skip = UINT32_MAX;
        t.ilimit = wobj;
        phase = 2;
        trace_begin(S, t, st);
        active = true;
        continue;
      }
      store_hit(w, p, t.h);
    }
  }
  flush_counters(cnt, rays, 0u, ts, 0u);
}

// Extension rays whose closest hit depends on the reference's object order
// (see scene_hit): the linear object loop.
__global__ void __launch_bounds__(128) wf_trace_fallback(DevScene S, WaveState w, DevCounters* cnt) {
  StackEntry lstack[kStackCap];
  StackEntry ltstack[kTlasStackCap];
  TravStats ts{0u, 0u, 0u, 0u};
  uint32_t const n = *w.n_fb;
  uint32_t const cap = w.cap;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t const p = w.fb_queue[i];
    Ray const r = make_ray(f3{w.ray[p], w.ray[cap + p], w.ray[2 * cap + p]},
                           f3{w.ray[3 * cap + p], w.ray[4 * cap + p], w.ray[5 * cap + p]});
    HitRec h;
    h.z = kFltMax;
    h.obj = UINT32_MAX;
    h.face = UINT32_MAX;
    h.b0 = h.b1 = h.b2 = 0.f;
    h.pl = f3{0.f, 0.f, 0.f};
    scene_hit<false>(S, r, h, UINT32_MAX, true, lstack, ltstack, ts);
    float* hp = w.hit;
    hp[0 * cap + p] = h.z;
    hp[1 * cap + p] = __uint_as_float(h.obj);
    hp[2 * cap + p] = __uint_as_float(h.face);
    hp[3 * cap + p] = h.b0;
    hp[4 * cap + p] = h.b1;
    hp[5 * cap + p] = h.b2;
    hp[6 * cap + p] = h.pl.x;
    hp[7 * cap + p] = h.pl.y;
    hp[8 * cap + p] = h.pl.z;
  }
  flush_counters(cnt, 0u, 0u, ts, 0u);
}

}  // namespace

// ---- shade ------------------------------------------------------------------------

template <int K>
__global__ void __launch_bounds__(128) wf_shade(DevScene S, RenderArgs a, WaveState w, DevCounters* cnt) {
  uint32_t const n = *w.n_in;
  uint32_t const cap = w.cap;
  float const omega = S.lambda_sup - S.lambda_inf;
  float const step = omega / float(K);
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t const i = base + threadIdx.x;
    bool const live = i < n;
    bool cont = false, shadow = false;
    uint32_t p = 0;
    f3 sp = f3{0.f, 0.f, 0.f}, sd = f3{0.f, 0.f, 1.f};
    float stmax = 0.f;
    uint32_t sskip = UINT32_MAX;
    f3 nd = f3{0.f, 0.f, 1.f}, np = f3{0.f, 0.f, 0.f};
    float lis_scale = 0.f, m_scale = 0.f;
    if (live) {
      p = w.q_in[i];
      HitRec h;
      h.obj = __float_as_uint(w.hit[cap + p]);
      if (h.obj != UINT32_MAX) {
        h.z = w.hit[p];
        h.face = __float_as_uint(w.hit[2 * cap + p]);
        h.b0 = w.hit[3 * cap + p];
        h.b1 = w.hit[4 * cap + p];
        h.b2 = w.hit[5 * cap + p];
        h.pl = f3{w.hit[6 * cap + p], w.hit[7 * cap + p], w.hit[8 * cap + p]};
        Ray const r = make_ray(f3{w.ray[p], w.ray[cap + p], w.ray[2 * cap + p]},
                               f3{w.ray[3 * cap + p], w.ray[4 * cap + p], w.ray[5 * cap + p]});
        HitInfo const H = finalize_hit(S, r, h);
        f3 const un = fnorm(r.u);
        f3 const o = f3{-un.x, -un.y, -un.z};
        f3 const nn = H.front ? H.F.z : neg3(H.F.z);
        const DevMaterial& m = S.mats[H.mat];
        float const hero = w.hero[p];
        if (m.type == LGPU_MAT_EMITTER || m.type == LGPU_MAT_DIREMITTER) {
          float g = 1.f;
          if (m.type == LGPU_MAT_DIREMITTER) {
            float const c = fdot(o, H.F.z);
            g = powf(c >= 0.f ? c : 0.f, m.specular);
          }
          for (int k = 0; k < K; k++) {
            float const x = lam_coord(S, hero_lambda(S, hero, step, k));
            w.acc[k * cap + p] += w.beta[k * cap + p] * (spec_at(S, m.spectrum[0], x) * g);
          }
        } else if (w.depth[p] <= a.max_scatter) {
          uint64_t rng = w.rng[p];
          uint32_t const li = uint32_t(lgpu_u64(&rng) % uint64_t(S.n_lights));
          float const prob_l = 1.f / float(S.n_lights);
          const lgpu_light& L = S.lights[li];
          // light sample without its visibility (the shadow kernel applies it)
          LightSample ls = sample_light_unoccluded(S, L, H, rng, stmax, sskip);
          float const x0 = lam_coord(S, hero);
          BsdfScalars const bl = bsdf_scalars(S, m, x0, ls.dir, o, nn, H.front);
          MatSample const ms = sample_material(S, m, x0, H, o, a.sample_p, rng);
          float w_L = 1.f, w_mat = 0.f;
          if (ms.ok) {
            float const p_L_mati = prob_for_light(S, L, H.p, ms.dir) * prob_l;
            float const p_mat_Li = prob_for_material(S, m, x0, H, ls.dir, o, a.sample_p);
            float const p_L_i = ls.prob * prob_l;
            w_L = p_L_i * p_L_i / (p_L_i * p_L_i + p_mat_Li * p_mat_Li);
            w_mat = ms.prob * ms.prob / (ms.prob * ms.prob + p_L_mati * p_L_mati);
          }
          lis_scale = ls.scale / (ls.prob * prob_l) * w_L;
          m_scale = ms.ok ? w_mat / ms.prob : 0.f;
          bool const needs_test = stmax >= 0.f;
          shadow = needs_test && lis_scale != 0.f;
          for (int k = 0; k < K; k++) {
            float const l = hero_lambda(S, hero, step, k);
            float const x = lam_coord(S, l);
            float const coef = bsdf_k(S, m, bl, x, l, H.front);
            float const rad = spec_at(S, L.spectrum, x);
            float const b = w.beta[k * cap + p];
            float const contrib = b * (rad * coef * lis_scale);
            if (!needs_test) w.acc[k * cap + p] += contrib;
            else w.s_contrib[k * cap + p] = contrib;  // slot p; gathered via s_path
            if (ms.ok) w.beta[k * cap + p] = b * (mat_mult_k(S, m, ms, x, l, H.front) * m_scale);
          }
          w.rng[p] = rng;
          sp = H.p;
          sd = ls.dir;
          cont = ms.ok;
          if (cont) {
            np = H.p;
            nd = ms.dir;
          }
        }
      }
    }
    // compacted appends: next-bounce queue, ended paths and shadow queue
    if (w.fin_list) {
      bool const ended = live && !cont;
      uint32_t const fo = warp_append(&w.ctl[2], ended);
      if (ended) w.fin_list[fo] = p;
    }
    uint32_t const qo = warp_append(w.n_out, cont);
    if (cont) {
      w.q_out[qo] = p;
      w.ray[0 * cap + p] = np.x;
      w.ray[1 * cap + p] = np.y;
      w.ray[2 * cap + p] = np.z;
      w.ray[3 * cap + p] = nd.x;
      w.ray[4 * cap + p] = nd.y;
      w.ray[5 * cap + p] = nd.z;
      w.depth[p] += 1;
    }
    uint32_t const so = warp_append(w.n_shadow, shadow);
    if (shadow) {
      w.s_path[so] = p;
      w.sray[0 * cap + so] = sp.x;
      w.sray[1 * cap + so] = sp.y;
      w.sray[2 * cap + so] = sp.z;
      w.sray[3 * cap + so] = sd.x;
      w.sray[4 * cap + so] = sd.y;
      w.sray[5 * cap + so] = sd.z;
      w.sray[6 * cap + so] = stmax;
      w.sray[7 * cap + so] = __uint_as_float(sskip);
    }
  }
  (void)cnt;
}

// ---- shadow -----------------------------------------------------------------------

template <int K>
__global__ void __launch_bounds__(128) wf_shadow(DevScene S, WaveState w, uint32_t flags, DevCounters* cnt) {
  extern __shared__ StackEntry smem_stack[];
  StackEntry lm[kLocalStack];
  StackEntry lstack[kStackCap];
  StackEntry ltstack[kTlasStackCap];
  SplitStack st{smem_stack + threadIdx.x, blockDim.x, lm, 0};
  TravStats ts{0u, 0u, 0u, 0u};
  uint32_t rays = 0;
  bool const ref_order = (flags & LGPU_FLAG_REFERENCE_ORDER) != 0;
  uint32_t const n = *w.n_shadow;
  uint32_t const cap = w.cap;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Ray const r = make_ray(f3{w.sray[i], w.sray[cap + i], w.sray[2 * cap + i]},
                           f3{w.sray[3 * cap + i], w.sray[4 * cap + i], w.sray[5 * cap + i]});
    HitRec h;
    h.z = w.sray[6 * cap + i];
    h.obj = UINT32_MAX;
    uint32_t const skip = __float_as_uint(w.sray[7 * cap + i]);
    bool const occ = scene_trace<true>(S, r, h, skip, ref_order, st, lstack, ltstack, ts);
    rays++;
    if (!occ) {
      uint32_t const p = w.s_path[i];
      for (int k = 0; k < K; k++) w.acc[k * cap + p] += w.s_contrib[k * cap + p];
    }
  }
  flush_counters(cnt, rays, 0u, ts, 0u);
}

// ---- film ---------------------------------------------------------------------------

template <int K>
__global__ void __launch_bounds__(256) wf_splat(DevScene S, WaveState w, DevCounters* cnt) {
  uint32_t nonfinite = 0;
  float const omega = S.lambda_sup - S.lambda_inf;
  float const step = omega / float(K);
  float const prob_l = 1.f / omega;
  for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < w.npix; pix += gridDim.x * blockDim.x) {
    float X = w.film[3 * pix], Y = w.film[3 * pix + 1], Z = w.film[3 * pix + 2];
    for (uint32_t s = 0; s < w.n_samples; s++) {
      uint32_t const p = s * w.npix + pix;
      float const hero = w.hero[p];
      float sx = 0.f, sy = 0.f, sz = 0.f;
      bool finite = true;
      for (int k = 0; k < K; k++) {
        float const val = w.acc[k * w.cap + p] / prob_l;
        finite = finite && isfinite(val);
        splat_xyz(S, hero_lambda(S, hero, step, k), val, sx, sy, sz);
      }
      nonfinite += finite ? 0u : 1u;
      X += sx;
      Y += sy;
      Z += sz;
    }
    w.film[3 * pix] = X;
    w.film[3 * pix + 1] = Y;
    w.film[3 * pix + 2] = Z;
  }
  TravStats const ts{0u, 0u, 0u, 0u};
  flush_counters(cnt, 0u, 0u, ts, nonfinite);
}

}  // namespace lgpu
