// lgpu_render.cuh — the render kernel, instantiated per hero-wavelength
// count in lgpu_render_k{4,8,16}.cu (separate units compile in parallel).
#pragma once

#include "lgpu_counters.cuh"
#include "lgpu_path.cuh"
#include "lgpu_wave.cuh"

namespace lgpu {

// Renderer::render (src/renderer.cpp:14-61) for a range of pixels: one
// thread per pixel, all of its samples, film accumulated as XYZ.
template <int K>
__global__ void __launch_bounds__(128) render_kernel(DevScene S, RenderArgs a, float* __restrict__ out,
                                                     DevCounters* cnt) {
  uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t rays = 0, nonfinite = 0, paths = 0;
  TravStats ts{0u, 0u, 0u, 0u};
  if (t < a.pixel_count) {
    uint32_t const pix = a.pixel_begin + t;
    uint32_t const W = uint32_t(S.cam.width), H = uint32_t(S.cam.height);
    uint32_t const i = pix / W, j = pix - i * W;
    float const omega = S.lambda_sup - S.lambda_inf;
    float const step = omega / float(K);
    float const prob_l = 1.f / omega;
    bool const ref_order = (a.flags & LGPU_FLAG_REFERENCE_ORDER) != 0;
    const lgpu_camera& C = S.cam;
    f3 const Fx = f3{C.base_x[0], C.base_x[1], C.base_x[2]};
    f3 const Fy = f3{C.base_y[0], C.base_y[1], C.base_y[2]};
    f3 const Fz = f3{C.base_z[0], C.base_z[1], C.base_z[2]};
    f3 const P = f3{C.pos[0], C.pos[1], C.pos[2]};
    Stacks st;
    float X = 0.f, Y = 0.f, Z = 0.f;
    uint64_t const stream = (uint64_t(a.stream_tag) << 32) | pix;
    for (uint32_t s = 0; s < a.spp; s++) {
      uint64_t rng = lgpu_path_state(a.seed, stream, uint64_t(a.spp_offset) + s);
      float const u = float(j) + lgpu_flt(&rng);
      float const v = float(i) + lgpu_flt(&rng);
      // sample::camera (cg.hpp:1534-1542)
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
      // sample::spectrum (cg.hpp:1517-1531)
      float const hero = S.lambda_inf + omega * lgpu_flt(&rng);
      float acc[K];
      PathCounters pc{0u, ts};
      trace_path<K>(S, make_ray(wkl, dir), hero, step, a.max_scatter, a.sample_p, ref_order, rng, acc, st,
                    pc);
      rays += pc.rays;
      ts = pc.ts;
      paths++;
      // addHeroλ(λ, Li/prob) (src/renderer.cpp:44)
      float sx = 0.f, sy = 0.f, sz = 0.f;
      bool finite = true;
#pragma unroll
      for (int k = 0; k < K; k++) {
        float const val = acc[k] / prob_l;
        finite = finite && isfinite(val);
        splat_xyz(S, hero_lambda(S, hero, step, k), val, sx, sy, sz);
      }
      nonfinite += finite ? 0u : 1u;
      X += sx;
      Y += sy;
      Z += sz;
    }
    // irradiance / (SPP*K), dotted with the CMFs times Δ, then XYZ2linRGB
    // (src/renderer.cpp:52-56, cg.hpp:144-148, 340-341)
    float const norm = float(a.spp * K);
    X = (X / norm) * S.lambda_delta;
    Y = (Y / norm) * S.lambda_delta;
    Z = (Z / norm) * S.lambda_delta;
    size_t const o = (size_t(H - i - 1) * W + j) * 3;
    out[o + 0] = 3.2404542f * X - 1.5371385f * Y - 0.4985314f * Z;
    out[o + 1] = -0.9692660f * X + 1.8760108f * Y + 0.0415560f * Z;
    out[o + 2] = 0.0556434f * X - 0.2040259f * Y + 1.0572252f * Z;
  }
  flush_counters(cnt, rays, paths, ts, nonfinite);
}

// Blocks per SM each wavefront kernel can keep resident (computed once per
// instantiation; the shading kernel per block size).
struct WaveOccupancy {
  uint32_t sms = 0;
  uint32_t trace, shadow, ptrace, pshadow, gen, fin, fb;
  uint32_t shade[kMaxShadeBlock / 32 + 1];  // 32, 64, ... threads per block (index block / 32)
};
constexpr size_t kTraceSmem = size_t(kSmemStack) * 128 * sizeof(StackEntry);

template <class F>
uint32_t blocks_per_sm(F kernel, int threads, size_t smem) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  return uint32_t(per_sm < 1 ? 1 : per_sm);
}

template <int K, class J>
const WaveOccupancy& wave_occupancy() {
  static WaveOccupancy o{};
  if (!o.sms) {
    size_t const smem = kTraceSmem;
    cudaFuncSetAttribute(wf_trace<J>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    cudaFuncSetAttribute(wf_shadow<K, J>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    cudaFuncSetAttribute(wf_trace_persistent<false, K, J>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(smem));
    cudaFuncSetAttribute(wf_trace_persistent<true, K, J>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(smem));
    o.trace = blocks_per_sm(wf_trace<J>, 128, smem);
    o.shadow = blocks_per_sm(wf_shadow<K, J>, 128, smem);
    o.ptrace = blocks_per_sm(wf_trace_persistent<false, K, J>, 128, smem);
    o.pshadow = blocks_per_sm(wf_trace_persistent<true, K, J>, 128, smem);
    o.gen = blocks_per_sm(wf_generate_stream<K, J>, 256, 0);
    o.fin = blocks_per_sm(wf_finish<K, J>, 256, 0);
    o.fb = blocks_per_sm(wf_trace_fallback<J>, 128, 0);
    for (uint32_t b = 1; b <= kMaxShadeBlock / 32; b++)
      o.shade[b] = blocks_per_sm(wf_shade<K, J, LGPU_MAT_LAMBERTIAN>, 32 * b, 0);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    o.sms = uint32_t(sms);
  }
  return o;
}

// Grids of one render: every SM filled to the kernel's occupancy limit, or
// to the configured cap for the persistent trace kernels.
struct WaveGrids {
  uint32_t trace, shade, shade_block, shadow, gen, ptrace, pshadow, fb, fin;
};

template <int K, class J>
WaveGrids wave_grids(const WaveConfig& cfg) {
  const WaveOccupancy& o = wave_occupancy<K, J>();
  uint32_t const sb = (cfg.shade_block >= 32 && cfg.shade_block <= kMaxShadeBlock && cfg.shade_block % 32 == 0)
                          ? cfg.shade_block
                          : 128;
  auto cap = [&](uint32_t per_sm) { return cfg.trace_per_sm && cfg.trace_per_sm < per_sm ? cfg.trace_per_sm : per_sm; };
  WaveGrids g;
  g.trace = o.sms * o.trace;
  g.shade_block = sb;
  g.shade = o.sms * o.shade[sb / 32];
  g.shadow = o.sms * o.shadow;
  g.gen = o.sms * o.gen;
  g.ptrace = o.sms * cap(o.ptrace);
  g.pshadow = o.sms * cap(o.pshadow);
  g.fb = o.sms * o.fb;
  g.fin = o.sms * o.fin;
  return g;
}

// Closest hits of the queue `w.in` (the instance BVH kernels, or the
// reference's linear object loop).
template <int K, class J>
void launch_closest(const J& jobs, const WaveState& w, const WaveGrids& g, bool linear, DevCounters* cnt,
                    cudaStream_t st) {
  if (linear) {
    wf_trace<J><<<g.trace, 128, kTraceSmem, st>>>(jobs, w, cnt);
  } else {
    wf_trace_persistent<false, K, J><<<g.ptrace, 128, kTraceSmem, st>>>(jobs, w, cnt);
    wf_trace_fallback<J><<<g.fb, 128, 0, st>>>(jobs, w, cnt);
  }
}

// Swaps the current and next queue, and the shadow contributions of this
// and the last iteration, after an iteration.
inline void swap_queues(WaveState& w) {
  PathBuf const pb = w.in;
  w.in = w.out;
  w.out = pb;
  uint32_t* const pc = w.n_in;
  w.n_in = w.n_out;
  w.n_out = pc;
  float* const sc = w.s_contrib;
  w.s_contrib = w.s_prev;
  w.s_prev = sc;
}

// The chunk is done when every work item was started and the queue is
// empty (the host copy of the counters, after the stream synchronised).
inline bool chunk_done(const WaveState& w, uint32_t total) {
  return w.h_ctl[kCtlNext] == total && w.h_ctl[w.n_in - w.ctl] == 0;
}

constexpr int kItersPerCheck = 4;

// Runs iterations of a chunk (issue(w) enqueues one iteration's kernels)
// until the chunk is done, reading the counters back every kItersPerCheck
// iterations.  With a graph cache and no per-kernel timing, the
// kItersPerCheck iterations and the counter readback are captured once as a
// CUDA graph and replayed; the graph's kernel arguments alternate the two
// queues, so the state is back in its starting parity after each replay.
template <class Issue>
cudaError_t run_iterations(WaveState& w, uint32_t total, cudaStream_t st, WaveLaunch* run, Issue issue) {
  size_t const ctl_bytes = kCtlWords * sizeof(uint32_t);
  bool graph = run->graph && run->cfg.graphs && !run->on;
  unsigned long long per_graph = 0;  // kernel launches in one replay
  if (graph) {
    cudaGraph_t gph = nullptr;
    unsigned long long const t0 = run->total;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      WaveState wc = w;
      for (int k = 0; k < kItersPerCheck; k++) {
        issue(wc);
        swap_queues(wc);
      }
      cudaMemcpyAsync(w.h_ctl, w.ctl, ctl_bytes, cudaMemcpyDeviceToHost, st);
      e = cudaStreamEndCapture(st, &gph);
    }
    per_graph = run->total - t0;
    run->total = t0;
    if (e == cudaSuccess) {
      GraphCache& gc = *run->graph;
      cudaGraphExecUpdateResultInfo info;
      if (!gc.exec || cudaGraphExecUpdate(gc.exec, gph, &info) != cudaSuccess) {
        cudaGetLastError();
        gc.release();
        e = cudaGraphInstantiate(&gc.exec, gph, 0);
      }
    }
    if (gph) cudaGraphDestroy(gph);
    if (e != cudaSuccess) {
      // capture is not possible on this stream (e.g. the legacy default
      // stream): launch the kernels one by one
      cudaGetLastError();
      graph = false;
    }
  }
  for (;;) {
    if (graph) {
      cudaError_t const e = cudaGraphLaunch(run->graph->exec, st);
      if (e != cudaSuccess) return e;
      run->graph_launches++;
      run->total += per_graph;
    } else {
      for (int k = 0; k < kItersPerCheck; k++) {
        issue(w);
        swap_queues(w);
      }
      cudaMemcpyAsync(w.h_ctl, w.ctl, ctl_bytes, cudaMemcpyDeviceToHost, st);
    }
    cudaError_t const e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    run->harvest();
    if (chunk_done(w, total)) return cudaSuccess;
  }
}

// One chunk of the streaming wavefront: work items [c0, c0 + total).
// Every iteration finishes the paths that ended in the last one, appends
// new paths behind the queue up to its capacity (plan + generate), then
// advances every queued path by one segment (trace, shade, shadow); the
// chunk's (sample, pixel) results are then added to the film.
template <int K, class J>
cudaError_t wave_chunk(const J& jobs, WaveState& w, uint64_t c0, uint32_t total, bool linear,
                       DevCounters* d_cnt, cudaStream_t st, WaveLaunch* run) {
  DevCounters* const c_closest = run->on ? d_cnt + 1 : d_cnt;
  DevCounters* const c_shadow = run->on ? d_cnt + 2 : d_cnt;
  WaveGrids const g = wave_grids<K, J>(run->cfg);
  w.c0 = c0;
  wf_stream_init<<<1, 32, 0, st>>>(w);
  run->total++;
  cudaError_t e = run_iterations(w, total, st, run, [&](const WaveState& wi) {
    wf_finish<K, J><<<g.fin, 256, 0, st>>>(jobs, wi, d_cnt);
    wf_plan<<<1, 1, 0, st>>>(wi, total);
    wf_generate_stream<K, J><<<g.gen, 256, 0, st>>>(jobs, wi, d_cnt);
    run->begin(0, st);
    launch_closest<K>(jobs, wi, g, linear, c_closest, st);
    run->end(0, st);
    run->begin(2, st);
    // one block per queue chunk, not persistent: a block's warps finish
    // their material-sorted groups at different times, and a persistent
    // block would hold the fast ones at the next chunk's sort barrier.
    // Three launches, each with one material type's code (the rest, Blinn,
    // thin film), so an SM's warps share their instructions; the first
    // lists the Blinn and thin-film hits for the other two.
    uint32_t const sg = (wi.cap + g.shade_block - 1) / g.shade_block;
    wf_shade<K, J, LGPU_MAT_LAMBERTIAN><<<sg, g.shade_block, 0, st>>>(jobs, wi, d_cnt);
    wf_shade<K, J, LGPU_MAT_BLINN><<<sg, g.shade_block, 0, st>>>(jobs, wi, d_cnt);
    wf_shade<K, J, LGPU_MAT_THINFILM><<<sg, g.shade_block, 0, st>>>(jobs, wi, d_cnt);
    run->end(2, st);
    run->begin(1, st);
    if (linear) wf_shadow<K, J><<<g.shadow, 128, kTraceSmem, st>>>(jobs, wi, c_shadow);
    else wf_trace_persistent<true, K, J><<<g.pshadow, 128, kTraceSmem, st>>>(jobs, wi, c_shadow);
    run->end(1, st);
    // finish, plan, generate, trace (+ fallback), shade (3), shadow
    run->total += linear ? 8 : 9;
  });
  if (e != cudaSuccess) return e;
  wf_finish<K, J><<<g.fin, 256, 0, st>>>(jobs, w, d_cnt);
  wf_reduce<J><<<(w.npix + 255) / 256, 256, 0, st>>>(jobs, w, c0 + total);
  run->total += 2;
  return cudaGetLastError();
}

template <int K, class J>
cudaError_t finalize_film(const J& jobs, const WaveState& w, cudaStream_t st, WaveLaunch* run) {
  wf_finalize<K, J><<<(w.npix + 255) / 256, 256, 0, st>>>(jobs, w);
  run->total++;
  cudaError_t e = cudaGetLastError();
  if (run->on && e == cudaSuccess) {
    e = cudaStreamSynchronize(st);
    run->harvest();
  }
  return e;
}

// The streaming wavefront over n_items work items of `jobs`, in chunks of
// at most chunk_items (the capacity of the (sample, pixel) film buffer).
template <int K, class J>
cudaError_t run_wave(const J& jobs, WaveState w, uint64_t n_items, uint64_t chunk_items, bool linear,
                     DevCounters* d_cnt, cudaStream_t st, WaveLaunch* run) {
  cudaError_t e = cudaMemsetAsync(w.film, 0, sizeof(float) * 3 * size_t(w.npix), st);
  if (e == cudaSuccess && w.film64) e = cudaMemsetAsync(w.film64, 0, sizeof(double) * 3 * size_t(w.npix), st);
  for (uint64_t c0 = 0; c0 < n_items && e == cudaSuccess; c0 += chunk_items) {
    uint32_t const total = uint32_t(n_items - c0 < chunk_items ? n_items - c0 : chunk_items);
    e = wave_chunk<K>(jobs, w, c0, total, linear, d_cnt, st, run);
  }
  if (e == cudaSuccess) e = finalize_film<K>(jobs, w, st, run);
  return e;
}

template <int K>
cudaError_t launch_render_k(const DevScene& S, const RenderArgs& a, WaveState* wave, float* d_out,
                            DevCounters* d_cnt, cudaStream_t st, WaveLaunch* run) {
  if (!wave) {
    uint32_t const blocks = (a.pixel_count + 127) / 128;
    render_kernel<K><<<blocks, 128, 0, st>>>(S, a, d_out, d_cnt);
    run->total++;
    return cudaGetLastError();
  }
  OneJob const jobs{S, a, wave->npix, d_out};
  // the instance BVH kernels, or the reference's linear object loop
  bool const linear = (a.flags & LGPU_FLAG_REFERENCE_ORDER) || S.n_objects <= 4;
  return run_wave<K>(jobs, *wave, uint64_t(wave->npix) * a.spp, uint64_t(wave->npix) * wave->n_samples,
                     linear, d_cnt, st, run);
}

template <int K>
cudaError_t launch_batch_k(const DevJob* d_jobs, const uint64_t* d_item_bases, const uint32_t* d_pix_bases,
                           uint32_t n_jobs, uint64_t n_items, uint64_t chunk_items, bool linear,
                           WaveState* wave, DevCounters* d_cnt, cudaStream_t st, WaveLaunch* run) {
  JobTable const jobs{d_jobs, d_item_bases, d_pix_bases, n_jobs};
  return run_wave<K>(jobs, *wave, n_items, chunk_items, linear, d_cnt, st, run);
}

}  // namespace lgpu
