// lgpu_trace.cu — ray-set queries (lgpu_trace_closest, lgpu_trace_any) run
// through the render's own traversal kernels.
//
// The rays of a query are put into a wavefront queue (closest-hit queries)
// or the shadow-ray queue (any-hit queries) of a WaveState of their own and
// traced by exactly the kernels a render launches for them:
// wf_trace_persistent<false> + wf_trace_fallback (instance BVH) or wf_trace
// (the reference's linear object loop) for closest hits, and
// wf_trace_persistent<true> or wf_shadow for shadow rays.  The hit records
// are then expanded to lgpu_hit with the same finalize_hit the shading uses.
#include "lgpu_render.cuh"

namespace lgpu {

namespace {

// The queue counters of one query chunk: n closest-hit rays in `in`, or n
// shadow rays; nothing fetched, nothing in the fallback list.
__global__ void trace_setup(WaveState w, uint32_t n, bool any) {
  if (threadIdx.x < kCtlWords) w.ctl[threadIdx.x] = 0u;
  __syncwarp();
  if (threadIdx.x == 0) {
    if (any) w.ctl[kCtlShadow] = n;
    else *w.n_in = n;
  }
}

// Rays (6 floats each, AoS) -> the queue's field-major layout; shadow rays
// also get their distance bound and object to skip.
__global__ void __launch_bounds__(256) trace_load(WaveState w, const float* __restrict__ rays,
                                                  const float* __restrict__ tmax,
                                                  const uint32_t* __restrict__ skip, uint32_t n, bool any) {
  uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float* const dst = any ? w.sray : w.in.ray;
  uint32_t const cap = w.cap;
#pragma unroll
  for (int c = 0; c < 6; c++) dst[c * cap + i] = rays[6 * size_t(i) + c];
  if (any) {
    dst[6 * cap + i] = tmax[i];
    dst[7 * cap + i] = __uint_as_float(skip[i]);
  }
}

// Hit records of the queue -> lgpu_hit (hitinfo, cg.hpp:1138-1149).
__global__ void __launch_bounds__(128) trace_store(DevScene S, WaveState w, uint32_t n,
                                                   lgpu_hit* __restrict__ out) {
  uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t const cap = w.cap;
  const float* hp = w.hit;
  HitRec h;
  h.z = hp[i];
  h.obj = __float_as_uint(hp[cap + i]);
  h.face = __float_as_uint(hp[2 * cap + i]);
  h.b0 = hp[3 * cap + i];
  h.b1 = hp[4 * cap + i];
  h.b2 = hp[5 * cap + i];
  h.pl = f3{hp[6 * cap + i], hp[7 * cap + i], hp[8 * cap + i]};
  lgpu_hit o;
  if (h.obj != UINT32_MAX) {
    HitInfo const H = finalize_hit(S, load_ray(w.in.ray, cap, i), h);
    o.t = H.z;
    o.obj = H.obj;
    o.face = H.face;
    o.mat = H.mat;
    o.p[0] = H.p.x; o.p[1] = H.p.y; o.p[2] = H.p.z;
    o.n[0] = H.F.z.x; o.n[1] = H.F.z.y; o.n[2] = H.F.z.z;
    o.gn[0] = H.gn.x; o.gn[1] = H.gn.y; o.gn[2] = H.gn.z;
    o.front = H.front ? 1u : 0u;
  } else {
    o.t = h.z;
    o.obj = UINT32_MAX;
    o.face = UINT32_MAX;
    o.mat = UINT32_MAX;
    for (int k = 0; k < 3; k++) o.p[k] = o.n[k] = o.gn[k] = 0.f;
    o.front = 0;
  }
  out[i] = o;
}

// Visibility bytes of the shadow queue -> the reference's return value
// (true = occluded).
__global__ void __launch_bounds__(256) trace_store_any(WaveState w, uint32_t n, uint8_t* __restrict__ out) {
  uint32_t const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = w.s_vis[i] ? 0 : 1;
}

// Grids of the traversal kernels: every SM filled to each kernel's
// occupancy limit (or the configured cap of the persistent kernels), as
// wave_grids sizes them for a render.
struct TraceGrids {
  uint32_t trace, shadow, ptrace, pshadow, fb;
};

TraceGrids trace_grids(const WaveConfig& cfg) {
  static uint32_t sms = 0, o_trace, o_shadow, o_ptrace, o_pshadow, o_fb;
  if (!sms) {
    o_trace = blocks_per_sm(wf_trace<OneJob>, 128, kTraceSmem);
    o_shadow = blocks_per_sm(wf_shadow<16, OneJob>, 128, kTraceSmem);
    o_ptrace = blocks_per_sm(wf_trace_persistent<false, 16, OneJob>, 128, kTraceSmem);
    o_pshadow = blocks_per_sm(wf_trace_persistent<true, 16, OneJob>, 128, kTraceSmem);
    o_fb = blocks_per_sm(wf_trace_fallback<OneJob>, 128, 0);
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    sms = uint32_t(n);
  }
  auto cap = [&](uint32_t per_sm) { return cfg.trace_per_sm && cfg.trace_per_sm < per_sm ? cfg.trace_per_sm : per_sm; };
  return TraceGrids{sms * o_trace, sms * o_shadow, sms * cap(o_ptrace), sms * cap(o_pshadow), sms * o_fb};
}

}  // namespace

size_t trace_wave_layout(uint8_t* base, uint32_t cap, WaveState& ws) {
  // the fields the traversal kernels touch; the rest stay null
  size_t off = 0;
  auto take = [&](size_t bytes) {
    uint8_t* const p = base ? base + off : nullptr;
    off += (bytes + 255) & ~size_t(255);
    return p;
  };
  ws = WaveState{};
  ws.cap = cap;
  ws.in.ray = reinterpret_cast<float*>(take(6 * sizeof(float) * size_t(cap)));
  ws.hit = reinterpret_cast<float*>(take(9 * sizeof(float) * size_t(cap)));
  ws.fb_queue = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * size_t(cap)));
  ws.sray = reinterpret_cast<float*>(take(8 * sizeof(float) * size_t(cap)));
  ws.s_vis = take(size_t(cap));
  ws.ctl = reinterpret_cast<uint32_t*>(take(kCtlWords * sizeof(uint32_t)));
  ws.n_in = ws.ctl + kCtlCountA;
  ws.n_out = ws.ctl + kCtlCountB;
  return off;
}

cudaError_t launch_trace_chunk(const DevScene& S, WaveState& w, const float* d_rays, const float* d_tmax,
                               const uint32_t* d_skip, uint32_t n, bool any, uint32_t flags,
                               lgpu_hit* d_hits, uint8_t* d_hit_any, const WaveConfig& cfg, DevCounters* d_cnt,
                               cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  RenderArgs a{};
  a.flags = flags & LGPU_FLAG_REFERENCE_ORDER;
  OneJob const jobs{S, a, 0u, nullptr};
  // the traversal kernels' code does not depend on the hero count K (a
  // template parameter they share with the shading); K = 16 as in renders
  // at the reference's spectral constants
  TraceGrids const g = trace_grids(cfg);
  bool const linear = (flags & LGPU_FLAG_REFERENCE_ORDER) || S.n_objects <= 4;
  trace_setup<<<1, 32, 0, st>>>(w, n, any);
  trace_load<<<(n + 255) / 256, 256, 0, st>>>(w, d_rays, d_tmax, d_skip, n, any);
  if (!any) {
    // the launches of launch_closest (lgpu_render.cuh)
    if (linear) {
      wf_trace<OneJob><<<g.trace, 128, kTraceSmem, st>>>(jobs, w, d_cnt);
    } else {
      wf_trace_persistent<false, 16, OneJob><<<g.ptrace, 128, kTraceSmem, st>>>(jobs, w, d_cnt);
      wf_trace_fallback<OneJob><<<g.fb, 128, 0, st>>>(jobs, w, d_cnt);
    }
    trace_store<<<(n + 127) / 128, 128, 0, st>>>(S, w, n, d_hits);
  } else {
    if (linear) wf_shadow<16, OneJob><<<g.shadow, 128, kTraceSmem, st>>>(jobs, w, d_cnt);
    else wf_trace_persistent<true, 16, OneJob><<<g.pshadow, 128, kTraceSmem, st>>>(jobs, w, d_cnt);
    trace_store_any<<<(n + 255) / 256, 256, 0, st>>>(w, n, d_hit_any);
  }
  return cudaGetLastError();
}

}  // namespace lgpu
