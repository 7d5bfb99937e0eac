// lgpu_wave.cuh — streaming wavefront path tracing.
//
// Paths in flight live in queue order: path i of the current queue keeps
// its state at index i of the `in` buffers (field-major, so a warp's access
// to one field is one coalesced transaction).  Each iteration
//
//   wf_finish<K>          ended paths of the last iteration (with the light
//                         sample of their last vertex if its shadow ray got
//                         through) -> XYZ of their (sample, pixel) film entry
//   wf_plan               how many new paths fit behind the queue
//   wf_generate_stream<K> camera ray + hero wavelengths of the new paths,
//                         appended to the queue
//   wf_trace_*            closest hit of every queued path
//   wf_shade<K>           adds the last vertex's light sample if its shadow
//                         ray got through; emitters, light sample -> shadow
//                         ray, material sample -> next ray; a continuing
//                         path is written to the next position of the `out`
//                         queue, an ended one to the ended list
//   wf_shadow / wf_trace_persistent<true>
//                         any-hit test of the shadow rays: one visibility
//                         byte per ray
//
// then the host swaps `in` and `out`.  No path keeps a fixed slot, so no
// access is scattered.  Each path draws its random numbers from its own
// counter-based stream in the order of Renderer::tracePath
// (src/renderer.cpp:64-146), and each (sample, pixel) result has its own
// film entry summed in sample order, so the image does not depend on how
// paths are scheduled.  Queue appends take one atomic per warp (ballot +
// popc).
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

__device__ __forceinline__ Ray load_ray(const float* ray, uint32_t cap, uint32_t i) {
  return make_ray(f3{ray[i], ray[cap + i], ray[2 * cap + i]},
                  f3{ray[3 * cap + i], ray[4 * cap + i], ray[5 * cap + i]});
}

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

__device__ __forceinline__ void clear_hit(HitRec& h, float z) {
  h.z = z;
  h.obj = UINT32_MAX;
  h.face = UINT32_MAX;
  h.b0 = h.b1 = h.b2 = 0.f;
  h.pl = f3{0.f, 0.f, 0.f};
}

// The non-template kernels get internal linkage: every translation unit
// that instantiates the renderer carries its own copy.
namespace {

// ---- streaming scheduler ------------------------------------------------------------

// Empty queue, no work handed out, nothing ended.
__global__ void wf_stream_init(WaveState w) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *w.n_in = 0;
    *w.n_out = 0;
    w.ctl[kCtlEnded] = 0;
    w.ctl[kCtlNext] = 0;
  }
}

// Runs after wf_finish: plans the next generate (as many new paths as fit
// behind the queue, up to the remaining work items) and clears the
// per-iteration counters.
__global__ void wf_plan(WaveState w, uint32_t total) {
  uint32_t const n_in = *w.n_in, next = w.ctl[kCtlNext];
  uint32_t const room = w.cap - n_in;
  uint32_t const left = total - next;
  uint32_t const n_new = room < left ? room : left;
  w.ctl[kCtlNew] = n_new;
  w.ctl[kCtlFirst] = next;
  w.ctl[kCtlPos] = n_in;
  w.ctl[kCtlNext] = next + n_new;
  *w.n_in = n_in + n_new;
  *w.n_out = 0;
  w.ctl[kCtlShadow] = 0;
  w.ctl[kCtlFetch] = 0;
  w.ctl[kCtlFetch + 1] = 0;
  w.ctl[kCtlFallback] = 0;
  w.ctl[kCtlEnded] = 0;
  w.ctl[kCtlListB] = 0;
  w.ctl[kCtlListT] = 0;
}

// Starts the planned paths at the end of the queue: work item q is sample
// q / npix of pixel q % npix (all pixels of one sample before the next).
// Camera ray and hero wavelength as sample::camera and sample::spectrum
// (cg.hpp:1534-1542, 1517-1531), random numbers drawn in the order of
// Renderer::render (src/renderer.cpp:33-41).
template <int K, class J>
__global__ void __launch_bounds__(256) wf_generate_stream(J jobs, WaveState w, DevCounters* cnt) {
  uint32_t const n_new = w.ctl[kCtlNew], first = w.ctl[kCtlFirst], pos = w.ctl[kCtlPos];
  uint32_t paths = 0;
  uint32_t const cap = w.cap;
  PathBuf const& in = w.in;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_new; k += gridDim.x * blockDim.x) {
    uint32_t const q = first + k;
    uint64_t const g = w.c0 + q;
    uint32_t const jb = jobs.job_of_item(g);
    const DevScene& S = jobs.scene(jb);
    const RenderArgs& a = jobs.args(jb);
    uint32_t const npix = jobs.npix_of(jb);
    uint64_t const l = g - jobs.item_base(jb);
    uint32_t const sample = uint32_t(l / npix);
    uint32_t const pix = jobs.frame_pixel(jb, uint32_t(l - uint64_t(sample) * npix));
    uint32_t const p = pos + k;
    float const omega = S.lambda_sup - S.lambda_inf;
    const lgpu_camera& C = S.cam;
    uint32_t const W = uint32_t(C.width);
    uint32_t const i = pix / W, j = pix - i * W;
    uint64_t rng = lgpu_path_state(a.seed, (uint64_t(a.stream_tag) << 32) | pix,
                                   uint64_t(a.spp_offset) + sample);
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
    in.sidx[p] = kNoShadow;
    if (J::kMulti) in.job[p] = jb;
    if (w.vis) w.vis[q] = 0;
    // no spectral state: a path at depth 0 has throughput 1 and no
    // radiance, which the shading kernel supplies (frame +1.8 % measured)
    paths++;
  }
  TravStats const ts{0u, 0u, 0u, 0u};
  flush_counters(cnt, 0u, paths, ts, 0u);
}

// Ended paths: radiance splatted to XYZ (addHeroλ(λ, Li/prob),
// src/renderer.cpp:44) into the path's (sample, pixel) film entry.
template <int K, class J>
__global__ void __launch_bounds__(256) wf_finish(J jobs, WaveState w, DevCounters* cnt) {
  uint32_t const n = w.ctl[kCtlEnded];
  uint32_t const cap = w.cap;
  uint32_t nonfinite = 0;
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const DevScene& S = jobs.scene(J::kMulti ? w.e_job[e] : 0u);
    float const omega = S.lambda_sup - S.lambda_inf;
    float const step = omega / float(K);
    float const prob_l = 1.f / omega;
    float const hero = w.e_hero[e];
    // the light sample of the path's last vertex, if its shadow ray got through
    uint32_t const sx_i = w.e_sidx[e];
    bool const lit = sx_i != kNoShadow && w.s_vis[sx_i];
    float sx = 0.f, sy = 0.f, sz = 0.f;
    bool finite = true;
#pragma unroll
    for (int k = 0; k < K; k++) {
      float acc = w.e_acc[k * cap + e];
      if (lit) acc += w.s_prev[k * cap + sx_i];
      if (w.ltot) w.ltot[size_t(w.e_item[e]) * K + k] = acc;
      float const val = acc / prob_l;
      finite = finite && isfinite(val);
      splat_xyz(S, hero_lambda(S, hero, step, k), val, sx, sy, sz);
    }
    nonfinite += finite ? 0u : 1u;
    size_t const o = 3 * size_t(w.e_item[e]);
    w.sbuf[o] = sx;
    w.sbuf[o + 1] = sy;
    w.sbuf[o + 2] = sz;
  }
  TravStats const ts{0u, 0u, 0u, 0u};
  flush_counters(cnt, 0u, 0u, ts, nonfinite);
}

// Film: per pixel, the (sample, pixel) entries of the chunk [w.c0, c1)
// added in sample order.
template <class J>
__global__ void __launch_bounds__(256) wf_reduce(J jobs, WaveState w, uint64_t c1) {
  for (uint32_t gp = blockIdx.x * blockDim.x + threadIdx.x; gp < w.npix; gp += gridDim.x * blockDim.x) {
    uint32_t const jb = jobs.job_of_pixel(gp);
    uint32_t const npix = jobs.npix_of(jb);
    uint64_t const base = jobs.item_base(jb) + (gp - jobs.pix_base(jb));
    uint32_t const spp = jobs.args(jb).spp;
    // samples s with w.c0 <= base + s * npix < c1
    uint64_t const lo = w.c0 > base ? (w.c0 - base + npix - 1) / npix : 0;
    uint64_t hi = c1 > base ? (c1 - base + npix - 1) / npix : 0;
    if (hi > spp) hi = spp;
    if (lo >= hi) continue;
    if (w.film64) {
      // the FP64 film: the same samples in the same order, summed in double
      double* const f = w.film64 + 3 * size_t(gp);
      double X = f[0], Y = f[1], Z = f[2];
      for (uint64_t s = lo; s < hi; s++) {
        size_t const o = 3 * size_t(base + s * npix - w.c0);
        X += double(w.sbuf[o]);
        Y += double(w.sbuf[o + 1]);
        Z += double(w.sbuf[o + 2]);
      }
      f[0] = X;
      f[1] = Y;
      f[2] = Z;
      continue;
    }
    float X = w.film[3 * size_t(gp)], Y = w.film[3 * size_t(gp) + 1], Z = w.film[3 * size_t(gp) + 2];
    for (uint64_t s = lo; s < hi; s++) {
      size_t const o = 3 * size_t(base + s * npix - w.c0);
      X += w.sbuf[o];
      Y += w.sbuf[o + 1];
      Z += w.sbuf[o + 2];
    }
    w.film[3 * size_t(gp)] = X;
    w.film[3 * size_t(gp) + 1] = Y;
    w.film[3 * size_t(gp) + 2] = Z;
  }
}

// XYZ film / (spp * K) * Δ -> linear BT.709 RGB in the reference's layout
// (row 0 at the top), src/renderer.cpp:52-56, cg.hpp:144-148, 340-341.
template <int K, class J>
__global__ void __launch_bounds__(256) wf_finalize(J jobs, WaveState w) {
  for (uint32_t gp = blockIdx.x * blockDim.x + threadIdx.x; gp < w.npix; gp += gridDim.x * blockDim.x) {
    uint32_t const jb = jobs.job_of_pixel(gp);
    const DevScene& S = jobs.scene(jb);
    uint32_t const pix = jobs.frame_pixel(jb, gp - jobs.pix_base(jb));
    uint32_t const W = uint32_t(S.cam.width), H = uint32_t(S.cam.height);
    uint32_t const i = pix / W, j = pix - i * W;
    if (w.film64) {
      // double throughout, into an output of doubles
      double const nd = double(jobs.args(jb).spp) * double(K);
      double const X = w.film64[3 * size_t(gp)] / nd * double(S.lambda_delta);
      double const Y = w.film64[3 * size_t(gp) + 1] / nd * double(S.lambda_delta);
      double const Z = w.film64[3 * size_t(gp) + 2] / nd * double(S.lambda_delta);
      double* o = reinterpret_cast<double*>(jobs.out_of(jb)) + (size_t(H - i - 1) * W + j) * 3;
      o[0] = 3.2404542 * X - 1.5371385 * Y - 0.4985314 * Z;
      o[1] = -0.9692660 * X + 1.8760108 * Y + 0.0415560 * Z;
      o[2] = 0.0556434 * X - 0.2040259 * Y + 1.0572252 * Z;
      continue;
    }
    float const norm = float(jobs.args(jb).spp) * float(K);
    float const X = (w.film[3 * size_t(gp)] / norm) * S.lambda_delta;
    float const Y = (w.film[3 * size_t(gp) + 1] / norm) * S.lambda_delta;
    float const Z = (w.film[3 * size_t(gp) + 2] / norm) * S.lambda_delta;
    float* out = jobs.out_of(jb) + (size_t(H - i - 1) * W + j) * 3;
    out[0] = 3.2404542f * X - 1.5371385f * Y - 0.4985314f * Z;
    out[1] = -0.9692660f * X + 1.8760108f * Y + 0.0415560f * Z;
    out[2] = 0.0556434f * X - 0.2040259f * Y + 1.0572252f * Z;
  }
}

// ---- trace ------------------------------------------------------------------------

// Closest hit of every queued path with one thread per ray (the reference's
// linear object loop, or the instance BVH).
template <class J>
__global__ void __launch_bounds__(128) wf_trace(J jobs, WaveState w, DevCounters* cnt) {
  extern __shared__ StackEntry smem_stack[];
  StackEntry lm[kLocalStack];
  StackEntry lstack[kStackCap];
  StackEntry ltstack[kTlasStackCap];
  SplitStack st{smem_stack + threadIdx.x, blockDim.x, lm, 0, 0u};
  TravStats ts{0u, 0u, 0u, 0u};
  uint32_t rays = 0;
  uint32_t const n = *w.n_in;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t const jb = J::kMulti ? w.in.job[i] : 0u;
    const DevScene& S = jobs.scene(jb);
    bool const ref_order = (jobs.args(jb).flags & LGPU_FLAG_REFERENCE_ORDER) != 0;
    Ray const r = load_ray(w.in.ray, w.cap, i);
    HitRec h;
    clear_hit(h, kFltMax);
    scene_trace<false>(S, r, h, UINT32_MAX, ref_order, st, lstack, ltstack, ts);
    rays++;
    store_hit(w, i, h);
  }
  ts.flags |= st.spill;
  flush_counters(cnt, rays, 0u, ts, 0u);
}

// Records whether shadow ray s reached its light.  Its radiance is added
// to the path by the next iteration's shading (or by wf_finish for an ended
// path), which reads the path's contributions in queue order, coalesced.
__device__ __forceinline__ void shadow_done(const WaveState& w, uint32_t s, bool unoccluded) {
  w.s_vis[s] = unoccluded ? 1 : 0;
  if (unoccluded && w.vis) w.vis[w.s_item[s]] |= 1ull << w.s_depth[s];
}

// Persistent instance-BVH traversal of the extension rays (ANY = false,
// the `in` queue, hit records out) or the shadow rays (ANY = true, one
// visibility byte each).  A lane that finishes its ray takes the next one;
// idle lanes are refilled together with one atomic per warp once kRefill of
// them are waiting (12 of 32: 8, 10 and 16 were slower).
constexpr int kRefill = 12;

// Occupancy (measured best): 7 blocks of 128 per SM (72 registers) for
// any-hit queries, 6 (80 registers) for closest-hit queries; the spills are a
// few bytes.
template <bool ANY, int K, class J>
__global__ void __launch_bounds__(128, ANY ? 7 : 6) wf_trace_persistent(J jobs, WaveState w, DevCounters* cnt) {
  extern __shared__ StackEntry smem_stack[];
  StackEntry lm[kLocalStack];
  SplitStack st{smem_stack + threadIdx.x, blockDim.x, lm, 0, 0u};
  __shared__ float wsave[9 * 128];  // launched with 128 threads
  st.ws = wsave + threadIdx.x;
  TravStats ts{0u, 0u, 0u, 0u};
  uint32_t rays = 0;
  uint32_t const n = ANY ? w.ctl[kCtlShadow] : *w.n_in;
  uint32_t* fetch = w.ctl + kCtlFetch + (ANY ? 1 : 0);
  uint32_t const cap = w.cap;
  unsigned const FULL = 0xFFFFFFFFu;
  int const lane = threadIdx.x & 31;
  TraceState t;
  bool active = false, exhausted = false;
  uint32_t idx = 0, wobj = 0, jb = 0;
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
          if (J::kMulti) jb = ANY ? w.s_job[my] : w.in.job[my];
          if (ANY) {
            t.w = load_ray(w.sray, cap, my);
            clear_hit(t.h, w.sray[6 * cap + my]);
            t.skip = __float_as_uint(w.sray[7 * cap + my]);
          } else {
            t.w = load_ray(w.in.ray, cap, my);
            clear_hit(t.h, kFltMax);
            t.skip = UINT32_MAX;
          }
          t.any = ANY;
          t.ilimit = UINT32_MAX;
          phase = 1;
          trace_begin(jobs.scene(jb), t, st);
          active = true;
          rays++;
        }
      }
    }
    if (__all_sync(FULL, !active)) {
      if (exhausted) break;
      continue;
    }
    if (active && trace_step<ANY>(jobs.scene(jb), t, st, ts)) {
      active = false;
      if (ANY) {
        shadow_done(w, idx, !t.hit_any);
        continue;
      }
      uint32_t const p = idx;
      if (phase == 2) {
        // an object below W's index is hit before the ray leaves W's bounds:
        // the reference skips W, so its answer is the closest hit without W
        if (t.hit_any) {
          t.w = load_ray(w.in.ray, cap, p);
          clear_hit(t.h, kFltMax);
          t.any = false;
          t.skip = wobj;
          t.ilimit = UINT32_MAX;
          phase = 3;
          trace_begin(jobs.scene(jb), t, st);
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
          w.fb_queue[atomicAdd(w.ctl + kCtlFallback, 1u)] = p;
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
        trace_begin(jobs.scene(jb), t, st);
        active = true;
        continue;
      }
      store_hit(w, p, t.h);
    }
  }
  ts.flags |= st.spill;
  flush_counters(cnt, rays, 0u, ts, 0u);
}

// Extension rays whose closest hit depends on the reference's object order
// (see scene_hit): the linear object loop, one warp per ray.  The lanes
// first test 32 objects at a time with an unbounded distance (the objects
// the ray cannot hit at all drop out); lane 0 then runs the reference's
// loop over the remaining ones in index order.  A launch has few such rays
// (about ten), so its time is the latency of one ray's loop, which the
// filter shortens from every object to the handful the ray can reach.
template <class J>
__global__ void __launch_bounds__(128) wf_trace_fallback(J jobs, WaveState w, DevCounters* cnt) {
  StackEntry lstack[kStackCap];
  TravStats ts{0u, 0u, 0u, 0u};
  uint32_t const n = w.ctl[kCtlFallback];
  uint32_t const lane = threadIdx.x & 31u;
  uint32_t const nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
    uint32_t const p = w.fb_queue[i];
    const DevScene& S = jobs.scene(J::kMulti ? w.in.job[p] : 0u);
    Ray const r = load_ray(w.in.ray, w.cap, p);
    HitRec h;
    clear_hit(h, kFltMax);
    h.inside = false;
    for (uint32_t base = 0; base < S.n_objects; base += 32) {
      uint32_t const o = base + lane;
      unsigned m = __ballot_sync(0xFFFFFFFFu, o < S.n_objects && object_may_hit(S, o, r));
      if (lane == 0)
        while (m) {
          uint32_t const b = uint32_t(__ffs(m) - 1);
          m &= m - 1u;
          object_hit<false>(S, base + b, r, h, lstack, ts, kRefOrder);
        }
      __syncwarp();
    }
    if (lane == 0) {
      store_hit(w, p, h);
      atomicAdd(&cnt->ordered, 1ull);
    }
  }
  flush_counters(cnt, 0u, 0u, ts, 0u);
}

}  // namespace

// ---- shade ------------------------------------------------------------------------

// Material sort within a block: the block's queue entries [base, base +
// blockDim.x) are handed to its threads grouped by what the shading kernel
// will do with them (miss, then material type, then past the queue end), so
// a warp's lanes take the same branch of the BSDF code.  A counting sort:
// per warp one ballot per group, a shared table of the warps' counts, and
// each thread's rank within its group.  Returns the entry for this thread.
constexpr int kSortGroups = 8;

template <class J>
__device__ __forceinline__ uint32_t material_order(const J& jobs, const WaveState& w, uint32_t base, uint32_t n,
                                                   uint32_t* group = nullptr) {
  __shared__ uint32_t counts[kSortGroups][kMaxShadeBlock / 32];
  __shared__ uint16_t perm[kMaxShadeBlock];
  __shared__ uint8_t groups[kMaxShadeBlock];
  uint32_t const t = threadIdx.x, lane = t & 31u, wid = t >> 5, nw = blockDim.x >> 5;
  uint32_t const q = base + t;
  uint32_t key = kSortGroups - 1;
  if (q < n) {
    uint32_t const obj = __float_as_uint(w.hit[w.cap + q]);
    if (obj == UINT32_MAX) {
      key = 0;
    } else {
      const DevScene& S = jobs.scene(J::kMulti ? w.in.job[q] : 0u);
      uint32_t const type = uint32_t(S.mats[S.objects[obj].mat].type);
      key = 1u + (type < kSortGroups - 3 ? type : kSortGroups - 3);
    }
  }
  unsigned mine = 0;
#pragma unroll
  for (int b = 0; b < kSortGroups; b++) {
    unsigned const m = __ballot_sync(0xFFFFFFFFu, key == uint32_t(b));
    if (key == uint32_t(b)) mine = m;
    if (lane == 0) counts[b][wid] = __popc(m);
  }
  __syncthreads();
  uint32_t pos = __popc(mine & ((1u << lane) - 1u));
  for (uint32_t b = 0; b < key; b++)
    for (uint32_t v = 0; v < nw; v++) pos += counts[b][v];
  for (uint32_t v = 0; v < wid; v++) pos += counts[key][v];
  perm[pos] = uint16_t(t);
  groups[pos] = uint8_t(key);
  __syncthreads();
  uint32_t const r = base + perm[t];
  if (group) *group = groups[t];
  __syncthreads();  // counts and perm are reused by the block's next chunk
  return r;
}

// After material_order: the block's Blinn entries are appended to the list
// at the front of w.shade_list, its thin-film entries to the list growing
// down from its end (both lists hold queue positions, together at most the
// queue's length).  A group is a contiguous range of the block's threads,
// so one atomic per list and block places it.
__device__ __forceinline__ void list_material_groups(const WaveState& w, uint32_t i, uint32_t group) {
  __shared__ uint32_t lbase[2];
  uint32_t const gb = 1u + LGPU_MAT_BLINN, gt = 1u + LGPU_MAT_THINFILM;
  uint32_t const below_b = uint32_t(__syncthreads_count(group < gb));
  uint32_t const cnt_b = uint32_t(__syncthreads_count(group == gb));
  uint32_t const below_t = uint32_t(__syncthreads_count(group < gt));
  uint32_t const cnt_t = uint32_t(__syncthreads_count(group == gt));
  if (threadIdx.x == 0) {
    lbase[0] = cnt_b ? atomicAdd(w.ctl + kCtlListB, cnt_b) : 0u;
    lbase[1] = cnt_t ? atomicAdd(w.ctl + kCtlListT, cnt_t) : 0u;
  }
  __syncthreads();
  if (group == gb) w.shade_list[lbase[0] + threadIdx.x - below_b] = i;
  if (group == gt) w.shade_list[w.cap - 1u - (lbase[1] + threadIdx.x - below_t)] = i;
  __syncthreads();  // lbase is reused by the block's next chunk
}

// One vertex of Renderer::tracePath (src/renderer.cpp:64-146) for every
// queued path: emitter hit (73-84), light importance sample with the MIS
// power heuristic (87-113, its visibility left to the shadow kernel),
// material importance sample with Russian roulette (115-143).
// MT < 0: every path; MT = LGPU_MAT_BLINN or LGPU_MAT_THINFILM: only the
// paths that hit that material (its code alone, the others' branches fold
// away); MT = LGPU_MAT_LAMBERTIAN: every other path (misses, emitters,
// Lambertian and unshaded materials).  The three specialised launches
// together shade every path once.
template <int MT>
__device__ __forceinline__ bool shade_group(uint32_t group) {
  if (MT < 0) return true;
  if (MT == LGPU_MAT_BLINN || MT == LGPU_MAT_THINFILM) return group == 1u + MT;
  return group != 1u + LGPU_MAT_BLINN && group != 1u + LGPU_MAT_THINFILM;
}

// Six blocks of 256 per SM (40 registers, with spills) for the first
// launch: the kernel waits on memory, and more warps hide it better than
// registers save spill traffic (4 blocks at 64 registers: +18 % shading
// time, 5: +2 %, 8: +5 %).  The list launches, whose warps are all busy,
// run 5 (48 registers; 6 and 4: +0.6 % and +0 % shading time).
template <int K, class J, int MT = -1>
__global__ void __launch_bounds__(kMaxShadeBlock, (MT == LGPU_MAT_BLINN || MT == LGPU_MAT_THINFILM) ? 5 : 6) wf_shade(J jobs, WaveState w, DevCounters* cnt) {
  uint32_t const n = *w.n_in;
  uint32_t const cap = w.cap;
  PathBuf const& in = w.in;
  PathBuf const& out = w.out;
  enum : int { kEnd = 0, kEmit = 1, kScatter = 2 };
  // the Blinn and thin-film launches run over their lists (dense warps)
  constexpr bool kList = MT == LGPU_MAT_BLINN || MT == LGPU_MAT_THINFILM;
  uint32_t const n_loop = kList ? w.ctl[MT == LGPU_MAT_BLINN ? kCtlListB : kCtlListT] : n;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n_loop; base += gridDim.x * blockDim.x) {
    uint32_t group = 0;
    // the first launch sorts each block's entries by material and appends
    // the Blinn and thin-film ones to the lists of the other two launches,
    // which shade them with full warps instead of the quarter of each block
    // that has their material (shading -24 % measured)
    uint32_t i;
    if (kList) {
      uint32_t const j = base + threadIdx.x;
      i = j < n_loop ? w.shade_list[MT == LGPU_MAT_BLINN ? j : cap - 1u - j] : UINT32_MAX;
      group = 1u + MT;
    } else {
      i = material_order(jobs, w, base, n, &group);
      if (MT == LGPU_MAT_LAMBERTIAN) list_material_groups(w, i, group);
    }
    bool const live = i < n && shade_group<MT>(group);
    uint32_t const jb = (J::kMulti && live) ? in.job[i] : 0u;
    const DevScene& S = jobs.scene(jb);
    const RenderArgs& a = jobs.args(jb);
    float const omega = S.lambda_sup - S.lambda_inf;
    float const step = omega / float(K);
    // the material as this launch sees it: a specialised launch knows its
    // type at compile time
    auto material = [&](uint32_t idx) {
      DevMaterial x = S.mats[idx];
      if (MT == LGPU_MAT_BLINN || MT == LGPU_MAT_THINFILM) x.type = MT;
      return x;
    };
    int kind = kEnd;
    bool cont = false, shadow = false, needs_test = false;
    f3 sp = f3{0.f, 0.f, 0.f}, sd = f3{0.f, 0.f, 1.f};
    float stmax = 0.f;
    uint32_t sskip = UINT32_MAX;
    f3 np = f3{0.f, 0.f, 0.f}, nd = f3{0.f, 0.f, 1.f};
    float lis_scale = 0.f, m_scale = 0.f, g_emit = 1.f, hero = 0.f;
    uint64_t rng = 0;
    uint32_t mat = 0, light = 0;
    bool front = true;
    MatSample ms;
    ms.ok = false;
    BsdfScalars bl{};
    if (live) {
      hero = in.hero[i];
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
        DevMaterial const m = material(mat);
        if (m.type == LGPU_MAT_EMITTER || m.type == LGPU_MAT_DIREMITTER) {
          kind = kEmit;
          if (m.type == LGPU_MAT_DIREMITTER) {
            float const c = fdot(o, H.F.z);
            g_emit = powf(c >= 0.f ? c : 0.f, m.specular);
          }
        } else if (in.depth[i] <= a.max_scatter) {
          kind = kScatter;
          rng = in.rng[i];
          light = uint32_t(lgpu_u64(&rng) % uint64_t(S.n_lights));
          float const prob_l = 1.f / float(S.n_lights);
          const lgpu_light& L = S.lights[light];
          // light sample without its visibility (the shadow kernel applies it)
          LightSample ls = sample_light_unoccluded(S, L, H, rng, stmax, sskip);
          float const x0 = lam_coord(S, hero);
          bl = bsdf_scalars(S, m, x0, ls.dir, o, nn, H.front);
          ms = sample_material(S, m, x0, H, o, a.sample_p, rng);
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
          needs_test = stmax >= 0.f;
          shadow = needs_test && lis_scale != 0.f;
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
    // compacted appends: next queue, ended list, shadow queue
    bool const ended = live && !cont;
    uint32_t const o_pos = warp_append(w.n_out, cont);
    uint32_t const e_pos = warp_append(w.ctl + kCtlEnded, ended);
    uint32_t const s_pos = warp_append(w.ctl + kCtlShadow, shadow);
    if (!live) continue;
    float* const acc_dst = cont ? out.acc + o_pos : w.e_acc + e_pos;
    DevMaterial const m = material(mat);
    // the light sample of the path's previous vertex, if its shadow ray got
    // through (recorded by the shadow kernel of the last iteration)
    uint32_t const prev_s = in.sidx[i];
    const float* const pend = (prev_s != kNoShadow && w.s_vis[prev_s]) ? w.s_prev + prev_s : nullptr;
    // a path at depth 0 starts with throughput 1 and no radiance (the
    // generate kernel writes neither)
    bool const fresh = in.depth[i] == 0;
    auto beta_k = [&](int k) { return fresh ? 1.f : in.beta[k * cap + i]; };
    auto acc_k = [&](int k) { return fresh ? 0.f : in.acc[k * cap + i]; };
    if (kind == kScatter) {
      const lgpu_light& L = S.lights[light];
      for (int k = 0; k < K; k++) {
        float const l = hero_lambda(S, hero, step, k);
        float const x = lam_coord(S, l);
        float const coef = bsdf_k(S, m, bl, x, l, front);
        float const rad = spec_at(S, L.spectrum, x);
        float const b = beta_k(k);
        float const contrib = b * (rad * coef * lis_scale);
        float acc = acc_k(k);
        if (pend) acc += pend[k * cap];
        if (!needs_test) acc += contrib;
        else if (shadow) w.s_contrib[k * cap + s_pos] = contrib;
        if (cont) out.beta[k * cap + o_pos] = b * (mat_mult_k(S, m, ms, x, l, front) * m_scale);
        acc_dst[k * cap] = acc;
      }
    } else if (kind == kEmit) {
      for (int k = 0; k < K; k++) {
        float const x = lam_coord(S, hero_lambda(S, hero, step, k));
        float acc = acc_k(k);
        if (pend) acc += pend[k * cap];
        acc_dst[k * cap] = acc + beta_k(k) * (spec_at(S, m.spectrum[0], x) * g_emit);
      }
    } else {
#pragma unroll
      for (int k = 0; k < K; k++) acc_dst[k * cap] = acc_k(k) + (pend ? pend[k * cap] : 0.f);
    }
    if (cont) {
      out.ray[0 * cap + o_pos] = np.x;
      out.ray[1 * cap + o_pos] = np.y;
      out.ray[2 * cap + o_pos] = np.z;
      out.ray[3 * cap + o_pos] = nd.x;
      out.ray[4 * cap + o_pos] = nd.y;
      out.ray[5 * cap + o_pos] = nd.z;
      out.rng[o_pos] = rng;
      out.hero[o_pos] = hero;
      out.depth[o_pos] = in.depth[i] + 1;
      out.item[o_pos] = in.item[i];
      out.sidx[o_pos] = shadow ? s_pos : kNoShadow;
      if (J::kMulti) out.job[o_pos] = jb;
    } else {
      w.e_hero[e_pos] = hero;
      w.e_item[e_pos] = in.item[i];
      w.e_sidx[e_pos] = shadow ? s_pos : kNoShadow;
      if (J::kMulti) w.e_job[e_pos] = jb;
    }
    if (shadow) {
      if (J::kMulti) w.s_job[s_pos] = jb;
      if (w.vis) {
        w.s_item[s_pos] = in.item[i];
        w.s_depth[s_pos] = in.depth[i];
      }
      w.sray[0 * cap + s_pos] = sp.x;
      w.sray[1 * cap + s_pos] = sp.y;
      w.sray[2 * cap + s_pos] = sp.z;
      w.sray[3 * cap + s_pos] = sd.x;
      w.sray[4 * cap + s_pos] = sd.y;
      w.sray[5 * cap + s_pos] = sd.z;
      w.sray[6 * cap + s_pos] = stmax;
      w.sray[7 * cap + s_pos] = __uint_as_float(sskip);
    }
  }
  (void)cnt;
}

// ---- shadow -----------------------------------------------------------------------

// Any-hit test of every shadow ray with one thread per ray.
template <int K, class J>
__global__ void __launch_bounds__(128) wf_shadow(J jobs, WaveState w, DevCounters* cnt) {
  extern __shared__ StackEntry smem_stack[];
  StackEntry lm[kLocalStack];
  StackEntry lstack[kStackCap];
  StackEntry ltstack[kTlasStackCap];
  SplitStack st{smem_stack + threadIdx.x, blockDim.x, lm, 0, 0u};
  TravStats ts{0u, 0u, 0u, 0u};
  uint32_t rays = 0;
  uint32_t const n = w.ctl[kCtlShadow];
  uint32_t const cap = w.cap;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t const jb = J::kMulti ? w.s_job[i] : 0u;
    const DevScene& S = jobs.scene(jb);
    bool const ref_order = (jobs.args(jb).flags & LGPU_FLAG_REFERENCE_ORDER) != 0;
    Ray const r = load_ray(w.sray, cap, i);
    HitRec h;
    clear_hit(h, w.sray[6 * cap + i]);
    uint32_t const skip = __float_as_uint(w.sray[7 * cap + i]);
    bool const occ = scene_trace<true>(S, r, h, skip, ref_order, st, lstack, ltstack, ts);
    rays++;
    shadow_done(w, i, !occ);
  }
  ts.flags |= st.spill;
  flush_counters(cnt, rays, 0u, ts, 0u);
}

}  // namespace lgpu
