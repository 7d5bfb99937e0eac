// lgpu_api.cu — the extern "C" entry points of include/lambda_gpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "lambda_gpu.h"
#include "lgpu_kernels.cuh"
#include "lgpu_layout.h"
#include "lgpu_layout_dev.h"

using namespace lgpu;

namespace {

template <class T>
struct DevArray {
  T* ptr = nullptr;
  size_t n = 0;    // elements in use
  size_t cap = 0;  // elements allocated
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = cap = 0;
  }
};

// The device arrays of one uploaded scene.
struct SceneSlot {
  DevScene S{};
  DevArray<DevObject> objects;
  DevArray<DevMesh> meshes;
  DevArray<WideNode> nodes;
  DevArray<TriSlot> tris;
  DevArray<FaceShade> shade;
  DevArray<float> spectra;
  DevArray<DevMaterial> mats;
  DevArray<lgpu_light> lights;
  DevArray<uint32_t> tlas_objects;
  DevArray<float> cmf;
  uint64_t bytes = 0;
  void release() {
    objects.release();
    meshes.release();
    nodes.release();
    tris.release();
    shade.release();
    spectra.release();
    mats.release();
    lights.release();
    tlas_objects.release();
    cmf.release();
    S = DevScene{};
    bytes = 0;
  }
};

}  // namespace

struct lgpu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  bool has_scene = false;
  DevScene S{};
  lgpu_stats stats{};
  // the scene table (lgpu_upload_scenes); S is a copy of slot 0's DevScene
  std::vector<SceneSlot> slots;
  HostLayout layout;  // host side of the last upload (its arrays are reused)
  // meshes laid out on the device (lgpu_layout_dev.cu): what to build, the
  // raw arrays of one mesh at a time, and the kernels' error word
  DeviceLayoutWork dev_layout;
  DevArray<uint8_t> raw;
  DevArray<uint32_t> layout_err;
  // meshes uploaded without a BVH: the trees built for them and the mesh
  // table pointing at them (build_missing_bvhs)
  std::vector<RefBvh> built;
  std::vector<lgpu_mesh> patched;
  // each mesh's traversal tree (build_traversal_trees): the caller's arrays
  // or a tree built here, kept until the next upload
  std::vector<TravTree> trav_views;
  std::vector<RefBvh> trav;
  std::vector<PrimBox> trav_boxes;
  std::vector<float> trav_cents;
  // batch tables (lgpu_render_batch)
  DevArray<DevJob> jobs;
  DevArray<uint64_t> job_items;
  DevArray<uint32_t> job_pixels;
  DevArray<float> batch_out;
  DevArray<float> adj_buf;
  // working buffers
  DevArray<float> out;
  // wavefront state (lgpu_wave.cuh), sized for the largest frame rendered
  DevArray<uint8_t> w_arena;
  uint32_t* h_ctl = nullptr;  // pinned
  DevArray<float> rays;
  DevArray<lgpu_hit> hits;
  // ray-set queries: their queue (lgpu_trace.cu) and shadow-ray inputs
  DevArray<uint8_t> trace_arena;
  DevArray<float> trace_tmax;
  DevArray<uint32_t> trace_skip;
  DevArray<uint8_t> trace_any;
  DevArray<lgpu_probe> probes;
  DevArray<lgpu_probe_result> probe_out;
  DevArray<double> partials;
  DevArray<float> tm_in, tm_out;
  DevArray<uint8_t> tm_24;
  DevCounters* counters = nullptr;  // 3 records: all kernels, closest-hit, shadow
  float* exposure = nullptr;
  WaveLaunch launch;
  bool events_ready = false;
  WaveConfig cfg;     // launch shape of the wavefront
  GraphCache graph;   // captured bounce stages
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaStream_t side = nullptr;  // batches: the megakernel jobs
  bool keep_counters = false;   // the counters were reset by the caller of a nested render

  void release_scene() {
    for (SceneSlot& sl : slots) sl.release();
    slots.clear();
    S = DevScene{};
    has_scene = false;
  }
};

namespace {

int fail(lgpu_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int cuda_fail(lgpu_ctx* ctx, cudaError_t e, const char* what) {
  int const code = (e == cudaErrorMemoryAllocation) ? LGPU_ERR_OUT_OF_MEMORY : LGPU_ERR_CUDA;
  return fail(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

// Copies h into d, reusing d's allocation when it is large enough.
template <class T, class Alloc>
cudaError_t upload(DevArray<T>& d, const std::vector<T, Alloc>& h, cudaStream_t st) {
  size_t const n = h.empty() ? 1 : h.size();
  cudaError_t e = cudaSuccess;
  if (!d.ptr || d.cap < n) {
    d.release();
    e = cudaMalloc(&d.ptr, n * sizeof(T));
    if (e != cudaSuccess) return e;
    d.cap = n;
  }
  d.n = h.size();
  if (!h.empty()) e = cudaMemcpyAsync(d.ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st);
  return e;
}

template <class T>
cudaError_t ensure(DevArray<T>& d, size_t n) {
  if (d.cap >= n && d.ptr) return cudaSuccess;
  d.release();
  cudaError_t const e = cudaMalloc(&d.ptr, (n ? n : 1) * sizeof(T));
  if (e == cudaSuccess) d.n = d.cap = n;
  return e;
}

int bind_device(lgpu_ctx* ctx) {
  cudaError_t const e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  return LGPU_OK;
}

// Work for a caller's stream runs on the context's own stream (where the
// bounce stages can be captured as a graph), ordered after what the caller
// enqueued before the call, and the caller's stream waits for it.
cudaError_t fork_from(lgpu_ctx* ctx, cudaStream_t user) {
  if (user == ctx->stream) return cudaSuccess;
  cudaError_t e = cudaEventRecord(ctx->ev_fork, user);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ctx->ev_fork, 0);
  return e;
}
cudaError_t join_to(lgpu_ctx* ctx, cudaStream_t user) {
  if (user == ctx->stream) return cudaSuccess;
  cudaError_t e = cudaEventRecord(ctx->ev_join, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(user, ctx->ev_join, 0);
  return e;
}

// Reads the device counters after a launch, updates the stats and reports
// device-side checks.
int collect(lgpu_ctx* ctx, const char* what, bool timed = false) {
  DevCounters r[3];
  cudaError_t e = cudaMemcpyAsync(r, ctx->counters, sizeof(r), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, what);
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) ctx->stats.last_kernel_ms = ms;
  DevCounters c = r[0];
  for (int k = 1; k < 3; k++) {
    c.rays += r[k].rays;
    c.paths += r[k].paths;
    c.nodes += r[k].nodes;
    c.tris += r[k].tris;
    c.insts += r[k].insts;
    c.flags |= r[k].flags;
    c.nonfinite += r[k].nonfinite;
    c.ordered += r[k].ordered;
  }
  ctx->stats.rays = c.rays;
  ctx->stats.paths = c.paths;
  ctx->stats.device_checks = c.flags & kTravOverflow;
  ctx->stats.node_tests = c.nodes;
  ctx->stats.tri_tests = c.tris;
  ctx->stats.inst_tests = c.insts;
  ctx->stats.nonfinite_paths = c.nonfinite;
  ctx->stats.order_rays = c.ordered;
  ctx->stats.local_stack = (c.flags & kTravLocalStack) ? 1u : 0u;
  ctx->stats.launches = uint32_t(ctx->launch.total);
  for (int k = 0; k < 3; k++) {
    ctx->stats.kernel_ms[k] = timed ? ctx->launch.ms[k] : 0.0;
    ctx->stats.kernel_launches[k] = timed ? ctx->launch.launches[k] : 0;
    // counters: [1] closest-hit, [2] shadow; shading does no traversal
    DevCounters const z{};
    const DevCounters& s = (timed && k < 2) ? r[k + 1] : z;
    ctx->stats.kernel_rays[k] = s.rays;
    ctx->stats.kernel_node_tests[k] = s.nodes;
    ctx->stats.kernel_tri_tests[k] = s.tris;
    ctx->stats.kernel_inst_tests[k] = s.insts;
  }
  if (c.flags & kTravOverflow)
    return fail(ctx, LGPU_ERR_DEVICE_CHECK,
                std::string(what) + ": a traversal stack bound was exceeded; results are incomplete");
  return LGPU_OK;
}

// Carves 256-byte aligned pieces out of one device allocation.
struct Carver {
  uint8_t* base;
  size_t off = 0;
  template <class T>
  T* take(size_t n) {
    T* const p = reinterpret_cast<T*>(base ? base + off : nullptr);
    off += (n * sizeof(T) + 255) & ~size_t(255);
    return p;
  }
};

// Lays out the wavefront buffers for queue capacity cap, K hero
// wavelengths, npix pixels and a chunk of sbuf_items work items; with
// base == nullptr it only counts the bytes.
size_t wave_layout(uint8_t* base, uint32_t cap, uint32_t K, uint32_t npix, uint64_t sbuf_items, bool batch,
                   bool adjoint, bool fp64, WaveState& ws) {
  Carver c{base};
  size_t const n = cap;
  for (PathBuf* pb : {&ws.in, &ws.out}) {
    pb->ray = c.take<float>(6 * n);
    pb->rng = c.take<uint64_t>(n);
    pb->hero = c.take<float>(n);
    pb->depth = c.take<uint32_t>(n);
    pb->item = c.take<uint32_t>(n);
    pb->job = batch ? c.take<uint32_t>(n) : nullptr;
    pb->beta = c.take<float>(size_t(K) * n);
    pb->acc = c.take<float>(size_t(K) * n);
    pb->gw = adjoint ? c.take<float>(size_t(K) * n) : nullptr;
    pb->sidx = c.take<uint32_t>(n);
  }
  ws.hit = c.take<float>(9 * n);
  ws.e_acc = c.take<float>(size_t(K) * n);
  ws.e_hero = c.take<float>(n);
  ws.e_item = c.take<uint32_t>(n);
  ws.e_job = batch ? c.take<uint32_t>(n) : nullptr;
  ws.sray = c.take<float>(8 * n);
  ws.e_sidx = c.take<uint32_t>(n);
  ws.s_contrib = c.take<float>(size_t(K) * n);
  ws.s_prev = c.take<float>(size_t(K) * n);
  ws.s_vis = c.take<uint8_t>(n);
  ws.s_job = batch ? c.take<uint32_t>(n) : nullptr;
  ws.fb_queue = c.take<uint32_t>(n);
  ws.shade_list = c.take<uint32_t>(n);
  ws.ctl = c.take<uint32_t>(kCtlWords);
  ws.film = c.take<float>(3 * size_t(npix));
  ws.film64 = fp64 ? c.take<double>(3 * size_t(npix)) : nullptr;
  ws.sbuf = c.take<float>(3 * size_t(sbuf_items));
  ws.ltot = adjoint ? c.take<float>(size_t(K) * sbuf_items) : nullptr;
  ws.vis = adjoint ? c.take<uint64_t>(sbuf_items) : nullptr;
  ws.s_item = adjoint ? c.take<uint32_t>(n) : nullptr;
  ws.s_depth = adjoint ? c.take<uint32_t>(n) : nullptr;
  return c.off;
}

// paths in flight: 2^24 (about 10.5 GB of path state at K = 16), fewer
// for small renders.  A deeper queue means fewer, longer launches per frame,
// so the launches' ramp-up and tail cost less of it (2^21: +10 % frame time,
// 2^23: +1 %)
constexpr uint64_t kQueueCap = uint64_t(1) << 24;
// the (sample, pixel) film buffer of one chunk stays under 8 GiB (of 180)
constexpr uint64_t kSbufBytes = uint64_t(1) << 33;

// Sizes the wavefront buffers for npix pixels, n_items work items in chunks
// of chunk_items, and fills ws.
int ensure_wave(lgpu_ctx* ctx, uint32_t npix, uint64_t n_items, uint64_t chunk_items, bool batch,
                WaveState& ws, bool adjoint = false, bool fp64 = false) {
  uint32_t const K = ctx->S.hero_k;
  uint64_t const qcap = ctx->cfg.queue_cap ? ctx->cfg.queue_cap : kQueueCap;
  uint32_t const cap = uint32_t(n_items < qcap ? n_items : qcap);
  size_t const bytes = wave_layout(nullptr, cap, K, npix, chunk_items, batch, adjoint, fp64, ws);
  cudaError_t const e = ensure(ctx->w_arena, bytes);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "wavefront buffers");
  wave_layout(ctx->w_arena.ptr, cap, K, npix, chunk_items, batch, adjoint, fp64, ws);
  ws.cap = cap;
  ws.npix = npix;
  ws.n_samples = 0;
  ws.c0 = 0;
  ws.n_in = ws.ctl + kCtlCountA;
  ws.n_out = ws.ctl + kCtlCountB;
  ws.h_ctl = ctx->h_ctl;
  return LGPU_OK;
}

// Creates the timing events on first use and resets the launch record.
int prepare_launch(lgpu_ctx* ctx, bool timing) {
  if (timing && !ctx->events_ready) {
    for (auto& k : ctx->launch.ev)
      for (auto& s : k)
        for (cudaEvent_t& ev : s)
          if (!ev && cudaEventCreate(&ev) != cudaSuccess) return fail(ctx, LGPU_ERR_CUDA, "timing events");
    ctx->events_ready = true;
  }
  ctx->launch.reset(timing);
  ctx->launch.cfg = ctx->cfg;
  ctx->launch.graph = &ctx->graph;
  return LGPU_OK;
}

RenderArgs render_args(const lgpu_render_params* p, const DevScene& S) {
  RenderArgs a{};
  a.spp = p->spp;
  a.max_scatter = p->max_scatterings;
  a.sample_p = p->sample_p;
  a.flags = p->flags;
  a.seed = p->seed;
  a.spp_offset = p->spp_offset;
  a.pixel_begin = 0;
  a.pixel_count = uint32_t(S.cam.width * S.cam.height);
  a.stream_tag = 0;
  return a;
}

// Renders scene S into d_out (device, linear RGB) on stream st.
int render_scene(lgpu_ctx* ctx, const DevScene& S, const lgpu_render_params* p, float* d_out,
                 cudaStream_t st) {
  if (!p || p->spp == 0) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "spp must be >= 1");
  bool const fp64 = (p->flags & LGPU_FLAG_FP64_FILM) != 0;
  if (fp64 && (p->flags & LGPU_FLAG_MEGAKERNEL))
    return fail(ctx, LGPU_ERR_UNSUPPORTED, "the FP64 film is a wavefront option (not with the megakernel)");
  RenderArgs const a = render_args(p, S);
  WaveState ws{};
  WaveState* wave = nullptr;
  if (!(p->flags & LGPU_FLAG_MEGAKERNEL)) {
    uint64_t const npix = a.pixel_count;
    uint64_t const max_ns = kSbufBytes / (12 * npix);
    uint32_t const ns = uint32_t(a.spp < max_ns ? a.spp : (max_ns ? max_ns : 1));
    int const r = ensure_wave(ctx, a.pixel_count, npix * a.spp, npix * ns, false, ws, false, fp64);
    if (r != LGPU_OK) return r;
    ws.n_samples = ns;
    wave = &ws;
  }
  if (int r = prepare_launch(ctx, (p->flags & LGPU_FLAG_KERNEL_TIMING) && wave)) return r;
  cudaError_t e = ctx->keep_counters ? cudaSuccess : cudaMemsetAsync(ctx->counters, 0, 3 * sizeof(DevCounters), st);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, st);
  if (e == cudaSuccess) e = launch_render(S, a, wave, d_out, ctx->counters, st, &ctx->launch);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "render launch");
  return LGPU_OK;
}

int render_impl(lgpu_ctx* ctx, const lgpu_render_params* p, float* d_out, cudaStream_t st) {
  if (!ctx->has_scene) return fail(ctx, LGPU_ERR_NO_SCENE, "no scene uploaded");
  return render_scene(ctx, ctx->S, p, d_out, st);
}

// The rectangle of a job in scene rows (x0, first scene row, width,
// height); false if it does not fit the frame.
bool job_rect(const lgpu_job& j, const lgpu_camera& c, uint32_t& x0, uint32_t& row0, uint32_t& w, uint32_t& h) {
  uint32_t const W = uint32_t(c.width), H = uint32_t(c.height);
  if (j.width == 0) {
    x0 = 0;
    row0 = 0;
    w = W;
    h = H;
    return true;
  }
  if (j.height == 0 || j.x0 >= W || j.y0 >= H || j.width > W - j.x0 || j.height > H - j.y0) return false;
  x0 = j.x0;
  w = j.width;
  h = j.height;
  row0 = H - j.y0 - j.height;  // output rows count from the top, scene rows from the bottom
  return true;
}

bool full_frame(const lgpu_job& j, const lgpu_camera& c) {
  return j.width == 0 || (j.x0 == 0 && j.y0 == 0 && j.width == uint32_t(c.width) && j.height == uint32_t(c.height));
}

int batch_impl(lgpu_ctx* ctx, const lgpu_job* jobs, uint32_t n, float* const* d_outs, cudaStream_t st);

// A batch split by the megakernel threshold: the small jobs render with the
// one-thread-per-pixel kernel on the side stream while the others take the
// wavefront on st.
int batch_split(lgpu_ctx* ctx, const lgpu_job* jobs, uint32_t n, float* const* d_outs, cudaStream_t st,
                const std::vector<uint32_t>& wave_jobs, const std::vector<uint32_t>& mega_jobs) {
  (void)n;
  if (!ctx->side) {
    cudaError_t const e = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "side stream");
  }
  if (int r = prepare_launch(ctx, false)) return r;
  cudaError_t e = cudaMemsetAsync(ctx->counters, 0, 3 * sizeof(DevCounters), st);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_fork, st);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0);
  for (uint32_t k : mega_jobs) {
    if (e != cudaSuccess) break;
    const DevScene& S = ctx->slots[jobs[k].scene].S;
    lgpu_render_params p = jobs[k].params;
    p.flags |= LGPU_FLAG_MEGAKERNEL;
    e = launch_render(S, render_args(&p, S), nullptr, d_outs[k], ctx->counters, ctx->side, &ctx->launch);
  }
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_join, ctx->side);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "megakernel jobs");
  unsigned long long const mega_launches = ctx->launch.total;
  int rc = LGPU_OK;
  if (!wave_jobs.empty()) {
    std::vector<lgpu_job> wj;
    std::vector<float*> wo;
    for (uint32_t k : wave_jobs) {
      wj.push_back(jobs[k]);
      wo.push_back(d_outs[k]);
    }
    // the counters were reset above and the megakernel jobs already count
    ctx->keep_counters = true;
    rc = batch_impl(ctx, wj.data(), uint32_t(wj.size()), wo.data(), st);
    ctx->keep_counters = false;
  }
  e = cudaStreamWaitEvent(st, ctx->ev_join, 0);
  ctx->launch.total += mega_launches;
  if (rc != LGPU_OK) return rc;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "megakernel join");
  return LGPU_OK;
}

// Renders the jobs (outputs d_outs, device) in one streaming wavefront; a
// single job takes the plain path.
int batch_impl(lgpu_ctx* ctx, const lgpu_job* jobs, uint32_t n, float* const* d_outs, cudaStream_t st) {
  if (!ctx->has_scene) return fail(ctx, LGPU_ERR_NO_SCENE, "no scene uploaded");
  bool timing = false, linear = false;
  for (uint32_t k = 0; k < n; k++) {
    if (jobs[k].scene >= ctx->slots.size())
      return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "job " + std::to_string(k) + ": no such scene");
    if (jobs[k].params.spp == 0)
      return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "job " + std::to_string(k) + ": spp must be >= 1");
    if (!d_outs[k]) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "job " + std::to_string(k) + ": null output");
    if (jobs[k].params.flags & LGPU_FLAG_FP64_FILM)
      return fail(ctx, LGPU_ERR_UNSUPPORTED, "job " + std::to_string(k) + ": the FP64 film is for plain renders");
    uint32_t x0, r0, tw, th;
    if (!job_rect(jobs[k], ctx->slots[jobs[k].scene].S.cam, x0, r0, tw, th))
      return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "job " + std::to_string(k) + ": rectangle outside the frame");
    timing = timing || (jobs[k].params.flags & LGPU_FLAG_KERNEL_TIMING);
    linear = linear || (jobs[k].params.flags & LGPU_FLAG_REFERENCE_ORDER);
  }
  if (n == 1 && full_frame(jobs[0], ctx->slots[jobs[0].scene].S.cam))
    return render_scene(ctx, ctx->slots[jobs[0].scene].S, &jobs[0].params, d_outs[0], st);
  // whole-frame jobs below the megakernel threshold run on the side stream
  std::vector<uint32_t> wave_jobs, mega_jobs;
  for (uint32_t k = 0; k < n; k++) {
    const lgpu_camera& c = ctx->slots[jobs[k].scene].S.cam;
    uint64_t const items = uint64_t(c.width) * c.height * jobs[k].params.spp;
    bool const mega = ctx->cfg.mega_items && items < ctx->cfg.mega_items && full_frame(jobs[k], c);
    (mega ? mega_jobs : wave_jobs).push_back(k);
  }
  if (!mega_jobs.empty()) return batch_split(ctx, jobs, n, d_outs, st, wave_jobs, mega_jobs);
  std::vector<DevJob> hj(n);
  std::vector<uint64_t> items(n + 1);
  std::vector<uint32_t> pixels(n + 1);
  uint64_t g = 0, px = 0;
  for (uint32_t k = 0; k < n; k++) {
    DevJob& d = hj[k];
    d.S = ctx->slots[jobs[k].scene].S;
    d.a = render_args(&jobs[k].params, d.S);
    uint32_t th = 0;
    job_rect(jobs[k], d.S.cam, d.col0, d.row0, d.tile_w, th);
    d.npix = d.tile_w * th;
    d.item_base = g;
    d.pix_base = uint32_t(px);
    d.out = d_outs[k];
    items[k] = g;
    pixels[k] = uint32_t(px);
    g += uint64_t(d.npix) * d.a.spp;
    px += d.npix;
    if (px >= (uint64_t(1) << 31))
      return fail(ctx, LGPU_ERR_TOO_LARGE, "a batch holds at most 2^31 pixels in all");
  }
  items[n] = g;
  pixels[n] = uint32_t(px);
  // a batch's film buffer may take 16 GiB (of 180), so that a typical batch
  // is one chunk with one drain at its end
  uint64_t const max_chunk = 2 * kSbufBytes / 12;
  uint64_t const chunk = g < max_chunk ? g : max_chunk;
  cudaError_t e = ensure(ctx->jobs, n);
  if (e == cudaSuccess) e = ensure(ctx->job_items, n + 1);
  if (e == cudaSuccess) e = ensure(ctx->job_pixels, n + 1);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch tables");
  e = cudaMemcpyAsync(ctx->jobs.ptr, hj.data(), n * sizeof(DevJob), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->job_items.ptr, items.data(), (n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->job_pixels.ptr, pixels.data(), (n + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice,
                        st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch tables");
  WaveState ws{};
  if (int r = ensure_wave(ctx, uint32_t(px), g, chunk, true, ws)) return r;
  if (int r = prepare_launch(ctx, timing)) return r;
  e = ctx->keep_counters ? cudaSuccess : cudaMemsetAsync(ctx->counters, 0, 3 * sizeof(DevCounters), st);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, st);
  if (e == cudaSuccess)
    e = launch_batch(ctx->S.hero_k, ctx->jobs.ptr, ctx->job_items.ptr, ctx->job_pixels.ptr, n, g, chunk, linear,
                     &ws, ctx->counters, st, &ctx->launch);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, st);
  // the host tables must outlive their asynchronous copies
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch launch");
  return LGPU_OK;
}

// Path-replay adjoint of a render of slot 0 (lgpu_adjoint.cuh).
int adjoint_impl(lgpu_ctx* ctx, const lgpu_render_params* p, const float* d_dimg, float* d_gspec, float* d_gmat,
                 float* d_img, cudaStream_t st) {
  if (!ctx->has_scene) return fail(ctx, LGPU_ERR_NO_SCENE, "no scene uploaded");
  if (!p || p->spp == 0) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "spp must be >= 1");
  if (p->max_scatterings > 62)
    return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "the adjoint records visibility for at most 63 vertices "
                                                "(max_scatterings <= 62)");
  if (p->flags & LGPU_FLAG_MEGAKERNEL)
    return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "the adjoint runs on the wavefront kernels only");
  if (p->flags & LGPU_FLAG_FP64_FILM)
    return fail(ctx, LGPU_ERR_UNSUPPORTED, "the adjoint's primal image is a float film");
  const DevScene& S = ctx->S;
  RenderArgs const a = render_args(p, S);
  uint64_t const npix = a.pixel_count;
  uint64_t const n_items = npix * a.spp;
  // per work item of a chunk: 12 B film entry, 4K B radiance, 8 B visibility
  uint64_t const per_item = 12 + 4ull * S.hero_k + 8;
  uint64_t const max_items = (uint64_t(1) << 34) / per_item;
  uint64_t const chunk = n_items < max_items ? n_items : max_items;
  WaveState ws{};
  if (int r = ensure_wave(ctx, a.pixel_count, n_items, chunk, false, ws, true)) return r;
  if (int r = prepare_launch(ctx, (p->flags & LGPU_FLAG_KERNEL_TIMING) != 0)) return r;
  size_t const n_spec = ctx->slots[0].spectra.n;
  cudaError_t e = cudaMemsetAsync(ctx->counters, 0, 3 * sizeof(DevCounters), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_gspec, 0, n_spec * sizeof(float), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_gmat, 0, 4 * size_t(S.n_materials) * sizeof(float), st);
  AdjointArgs const g{d_dimg, d_gspec, d_gmat};
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, st);
  if (e == cudaSuccess) e = launch_adjoint(S.hero_k, S, a, &ws, chunk, d_img, g, ctx->counters, st, &ctx->launch);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint launch");
  return LGPU_OK;
}

bool batch_timing(const lgpu_job* jobs, uint32_t n) {
  for (uint32_t k = 0; k < n; k++)
    if ((jobs[k].params.flags & LGPU_FLAG_KERNEL_TIMING) && !(n == 1 && (jobs[k].params.flags & LGPU_FLAG_MEGAKERNEL)))
      return true;
  return false;
}

// per-kernel timing applies to the wavefront kernels only
bool timing_requested(const lgpu_render_params* p) {
  return (p->flags & LGPU_FLAG_KERNEL_TIMING) && !(p->flags & LGPU_FLAG_MEGAKERNEL);
}

// Lays out one scene on the host and copies it into a scene slot.
// The raw arrays of the meshes of the last device-layout upload, one mesh
// at a time through ctx->raw (256-byte aligned pieces), and the kernels
// that lay them out into the slot's node, triangle and shading arrays.
int build_meshes_on_device(lgpu_ctx* ctx, SceneSlot& sl, const lgpu_scene& scene, uint64_t& bytes) {
  const DeviceLayoutWork& W = ctx->dev_layout;
  cudaStream_t const st = ctx->stream;
  // a job's tree: the mesh's own BVH, or its traversal tree
  struct Tree {
    uint32_t n_nodes, n_bbs, n_prims;
    const uint32_t* nodes;
    const float* bbs;
    const uint32_t* prims;
  };
  auto tree_of = [&](const DeviceMeshJob& j) {
    const lgpu_mesh& m = scene.meshes[j.mesh];
    if (!j.tree) return Tree{m.n_nodes, m.n_bbs, m.n_prim_idxs, m.nodes, m.bbs, m.prim_idxs};
    return Tree{j.tree->n_nodes, j.tree->n_bbs, j.tree->n_prims, j.tree->nodes, j.tree->bbs, j.tree->prims};
  };
  auto pieces = [](const lgpu_mesh& m, const Tree& T, size_t (&sz)[8]) {
    sz[0] = 12 * size_t(m.n_positions);
    sz[1] = 12 * size_t(m.n_normals);
    sz[2] = 12 * size_t(m.n_faces);
    sz[3] = 4 * size_t(m.f_stride) * m.n_faces;
    sz[4] = 8 * size_t(T.n_nodes);
    sz[5] = 192 * size_t(T.n_bbs);
    sz[6] = 4 * size_t(T.n_prims);
    sz[7] = 4 * size_t(T.n_nodes);
    size_t t = 0;
    for (size_t x : sz) t += (x + 255) & ~size_t(255);
    return t;
  };
  size_t most = 0;
  for (const DeviceMeshJob& j : W.jobs) {
    size_t sz[8];
    most = std::max(most, pieces(scene.meshes[j.mesh], tree_of(j), sz));
  }
  cudaError_t e = ensure(ctx->raw, most);
  if (e == cudaSuccess) e = ensure(ctx->layout_err, 1);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->layout_err.ptr, 0xFF, sizeof(uint32_t), st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "mesh layout buffers");
  for (const DeviceMeshJob& j : W.jobs) {
    const lgpu_mesh& m = scene.meshes[j.mesh];
    Tree const T = tree_of(j);
    size_t sz[8];
    pieces(m, T, sz);
    const void* src[8] = {m.V, m.N, m.GN, m.F, T.nodes, T.bbs, T.prims, W.childref.data() + j.childref_off};
    void* dst[8];
    size_t off = 0;
    for (int k = 0; k < 8 && e == cudaSuccess; k++) {
      dst[k] = ctx->raw.ptr + off;
      off += (sz[k] + 255) & ~size_t(255);
      // a traversal tree's job follows its mesh's own job: the mesh's
      // arrays (pieces 0-3, at the same offsets) are still in place
      if (j.tree && k < 4) continue;
      if (sz[k]) e = cudaMemcpyAsync(dst[k], src[k], sz[k], cudaMemcpyHostToDevice, st);
      bytes += sz[k];
    }
    MeshRaw const r{static_cast<const float*>(dst[0]), static_cast<const float*>(dst[1]),
                    static_cast<const float*>(dst[2]), static_cast<const uint32_t*>(dst[3]),
                    static_cast<const uint32_t*>(dst[4]), static_cast<const float*>(dst[5]),
                    static_cast<const uint32_t*>(dst[6]), static_cast<const uint32_t*>(dst[7]),
                    m.n_positions, m.n_normals, m.n_faces, m.f_stride, T.n_nodes, T.n_prims};
    if (e == cudaSuccess)
      e = build_mesh_layout(r, j.mesh, sl.nodes.ptr, sl.tris.ptr + j.slot_base,
                            j.tree ? nullptr : sl.shade.ptr + j.face_base, ctx->layout_err.ptr, st);
    // the next mesh's copies reuse ctx->raw: stream order puts them after
    // these kernels; the host's pageable copies return once staged
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "mesh layout");
  return LGPU_OK;
}

// Meshes passed without their BVH (nodes, bbs and prim_idxs all NULL) get
// it built here on the device, bit-identical to bvh::build (cg.hpp:632-749);
// `out` is the scene with those meshes pointing at the built trees, kept in
// ctx->built until the next upload.
int build_missing_bvhs(lgpu_ctx* ctx, const lgpu_scene& in, lgpu_scene& out) {
  out = in;
  ctx->built.clear();
  ctx->patched.clear();
  bool any = false;
  for (uint32_t mi = 0; mi < in.n_meshes && in.meshes; mi++) {
    const lgpu_mesh& m = in.meshes[mi];
    any = any || (!m.nodes && !m.bbs && !m.prim_idxs);
  }
  if (!any) return LGPU_OK;
  ctx->built.resize(in.n_meshes);
  ctx->patched.assign(in.meshes, in.meshes + in.n_meshes);
  for (uint32_t mi = 0; mi < in.n_meshes; mi++) {
    lgpu_mesh& m = ctx->patched[mi];
    if (m.nodes || m.bbs || m.prim_idxs) continue;
    std::string const what = "mesh " + std::to_string(mi) + ": ";
    if (!m.V || !m.F || m.f_stride < 3 || m.n_faces == 0)
      return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "incomplete mesh " + std::to_string(mi));
    for (uint32_t f = 0; f < m.n_faces; f++)
      for (int k = 0; k < 3; k++)
        if (m.F[size_t(f) * m.f_stride + k] >= m.n_positions)
          return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "face index out of range in mesh " + std::to_string(mi));
    for (size_t i = 0; i < 3 * size_t(m.n_positions); i++)
      if (!std::isfinite(m.V[i]))
        return fail(ctx, LGPU_ERR_INVALID_ARGUMENT,
                    what + "vertex " + std::to_string(i / 3) + " is not finite (no BVH can be built)");
    RefBvh& B = ctx->built[mi];
    cudaError_t e;
    try {
      e = build_bvh_device(m.V, m.n_positions, m.F, m.f_stride, m.n_faces, B, ctx->stream);
    } catch (const std::bad_alloc&) {
      return fail(ctx, LGPU_ERR_OUT_OF_MEMORY, what + "host memory for the BVH");
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "device BVH build");
    m.nodes = B.nodes.data();
    m.bbs = B.bbs.data();
    m.prim_idxs = B.prim_idxs.data();
    m.n_nodes = B.n_nodes;
    m.n_bbs = uint32_t(B.bbs.size() / 48);
    m.n_prim_idxs = uint32_t(B.prim_idxs.size());
  }
  out.meshes = ctx->patched.data();
  return LGPU_OK;
}

// Each mesh's traversal tree, unless the scene keeps the reference's trees:
// the caller's (lgpu_mesh::trav_*), or one built here (build_sah_bvh, leaves
// of at most 2 faces: 1, 3, 4 and 8 were slower).  A mesh whose faces index
// outside its positions, or whose triangles are not finite, gets none here:
// the layout reports a bad index, and the reference's tree serves a
// non-finite mesh as the reference's own traversal would.
int build_traversal_trees(lgpu_ctx* ctx, const lgpu_scene& sc) {
  ctx->trav_views.assign(sc.n_meshes, TravTree{});
  ctx->trav.resize(sc.n_meshes);
  if ((sc.flags & LGPU_SCENE_REFERENCE_BVH) || !sc.meshes) return LGPU_OK;
  for (uint32_t mi = 0; mi < sc.n_meshes; mi++) {
    const lgpu_mesh& m = sc.meshes[mi];
    bool const any = m.trav_nodes || m.trav_bbs || m.trav_prim_idxs;
    if (any) {
      if (!m.trav_nodes || !m.trav_bbs || !m.trav_prim_idxs || m.n_trav_nodes == 0)
        return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "incomplete traversal tree of mesh " + std::to_string(mi));
      ctx->trav_views[mi] = TravTree{m.n_trav_nodes, m.n_trav_bbs, m.n_trav_prim_idxs,
                                     m.trav_nodes,   m.trav_bbs,   m.trav_prim_idxs};
      continue;
    }
    RefBvh& T = ctx->trav[mi];
    T.n_nodes = 0;
    if (!m.V || !m.F || m.f_stride < 3 || m.n_faces == 0) continue;
    bool ok = true;
    for (size_t f = 0; f < m.n_faces && ok; f++)
      for (int k = 0; k < 3; k++) ok = ok && m.F[f * m.f_stride + k] < m.n_positions;
    if (!ok) continue;
    try {
      triangle_prims(m.V, m.F, m.f_stride, m.n_faces, ctx->trav_boxes, ctx->trav_cents);
      for (const PrimBox& b : ctx->trav_boxes)
        for (int k = 0; k < 3 && ok; k++) ok = std::isfinite(b.inf[k]) && std::isfinite(b.sup[k]);
      for (size_t i = 0; i < ctx->trav_cents.size() && ok; i++) ok = std::isfinite(ctx->trav_cents[i]);
      if (!ok) continue;
      build_sah_bvh(m.n_faces, ctx->trav_boxes.data(), ctx->trav_cents.data(), T, 2);
    } catch (const std::exception&) {
      T = RefBvh{};  // no host memory or threads: the reference's tree serves
      continue;
    }
    ctx->trav_views[mi] = TravTree{T.n_nodes, uint32_t(T.bbs.size() / 48), uint32_t(T.prim_idxs.size()),
                                   T.nodes.data(), T.bbs.data(), T.prim_idxs.data()};
  }
  return LGPU_OK;
}

int upload_slot(lgpu_ctx* ctx, SceneSlot& sl, const lgpu_scene& scene_in) {
  lgpu_scene scene;
  if (int r = build_missing_bvhs(ctx, scene_in, scene)) return r;
  if (int r = build_traversal_trees(ctx, scene)) return r;
  HostLayout& L = ctx->layout;
  std::string err;
  bool const on_device = !(scene.flags & LGPU_SCENE_HOST_LAYOUT);
  DeviceLayoutWork& W = ctx->dev_layout;
  int const rc = make_layout(scene, L, err, on_device ? &W : nullptr, &ctx->trav_views);
  if (rc != LGPU_OK) return fail(ctx, rc, err);
  cudaStream_t const st = ctx->stream;
  uint64_t bytes = 0;
  cudaError_t e = upload(sl.objects, L.objects, st);
  if (e == cudaSuccess) e = upload(sl.meshes, L.meshes, st);
  if (on_device) {
    // the meshes' nodes first (built on the device), then the instance BVH's
    size_t const n_nodes = size_t(W.mesh_nodes) + L.nodes.size();
    if (e == cudaSuccess) e = ensure(sl.nodes, n_nodes);
    if (e == cudaSuccess) e = ensure(sl.tris, W.mesh_slots);
    if (e == cudaSuccess) e = ensure(sl.shade, W.mesh_faces);
    sl.nodes.n = n_nodes;
    sl.tris.n = W.mesh_slots;
    sl.shade.n = W.mesh_faces;
    if (e == cudaSuccess && !L.nodes.empty())
      e = cudaMemcpyAsync(sl.nodes.ptr + W.mesh_nodes, L.nodes.data(), L.nodes.size() * sizeof(WideNode),
                          cudaMemcpyHostToDevice, st);
    bytes += L.nodes.size() * sizeof(WideNode);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "scene upload");
    if (int r = build_meshes_on_device(ctx, sl, scene, bytes)) return r;
  } else {
    if (e == cudaSuccess) e = upload(sl.nodes, L.nodes, st);
    if (e == cudaSuccess) e = upload(sl.tris, L.tris, st);
    if (e == cudaSuccess) e = upload(sl.shade, L.shade, st);
    bytes += L.nodes.size() * sizeof(WideNode) + L.tris.size() * sizeof(TriSlot) +
             L.shade.size() * sizeof(FaceShade);
  }
  if (e == cudaSuccess) e = upload(sl.spectra, L.spectra, st);
  if (e == cudaSuccess) e = upload(sl.mats, L.mats, st);
  if (e == cudaSuccess) e = upload(sl.lights, L.lights, st);
  if (e == cudaSuccess) e = upload(sl.tlas_objects, L.tlas_objects, st);
  if (e == cudaSuccess) e = upload(sl.cmf, L.cmf, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "scene upload");
  if (on_device) {
    uint32_t code = UINT32_MAX;
    e = cudaMemcpy(&code, ctx->layout_err.ptr, sizeof(code), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "scene upload");
    if (code != UINT32_MAX) {
      uint32_t const mi = code / 4;
      return fail(ctx, LGPU_ERR_INVALID_ARGUMENT,
                  (code % 4 == 1 ? "face index out of range in mesh " : "BVH primitive index out of range in mesh ") +
                      std::to_string(mi));
    }
  }
  bytes += L.objects.size() * sizeof(DevObject) + L.meshes.size() * sizeof(DevMesh) +
           L.spectra.size() * sizeof(float) + L.mats.size() * sizeof(DevMaterial) +
           L.lights.size() * sizeof(lgpu_light) + L.tlas_objects.size() * sizeof(uint32_t) +
           L.cmf.size() * sizeof(float);
  DevScene& S = sl.S;
  S = DevScene{};
  S.objects = sl.objects.ptr;
  S.meshes = sl.meshes.ptr;
  S.nodes = sl.nodes.ptr;
  S.tris = sl.tris.ptr;
  S.shade = sl.shade.ptr;
  S.spectra = sl.spectra.ptr;
  S.mats = sl.mats.ptr;
  S.lights = sl.lights.ptr;
  S.tlas_objects = sl.tlas_objects.ptr;
  S.n_objects = scene.n_objects;
  S.n_meshes = scene.n_meshes;
  S.n_materials = scene.n_materials;
  S.n_lights = scene.n_lights;
  S.tlas_root = L.tlas_root;
  S.max_stack = L.max_stack;
  S.tlas_max_stack = L.tlas_max_stack;
  S.n_bins = scene.spec.n_bins;
  S.hero_k = scene.spec.hero_k;
  S.lambda_inf = scene.spec.lambda_inf;
  S.lambda_sup = scene.spec.lambda_sup;
  // coefficientλ::Δ = (sup-inf)/(n-1) (cg.hpp:246)
  S.lambda_delta = (S.lambda_sup - S.lambda_inf) / float(S.n_bins - 1);
  S.cmf = sl.cmf.ptr;
  S.cam = scene.cam;
  std::memcpy(S.tlas_bounds, L.tlas_bounds, sizeof(S.tlas_bounds));
  if (L.max_stack > ctx->stats.max_stack) ctx->stats.max_stack = L.max_stack;
  sl.bytes = bytes;
  return LGPU_OK;
}

}  // namespace

extern "C" {

int lgpu_abi_version(void) { return LGPU_ABI_VERSION; }

int lgpu_create(int device, lgpu_ctx** out) {
  if (!out) return LGPU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return LGPU_ERR_NO_DEVICE;
  if (device < 0 || device >= n) return LGPU_ERR_INVALID_ARGUMENT;
  lgpu_ctx* ctx = new (std::nothrow) lgpu_ctx;
  if (!ctx) return LGPU_ERR_OUT_OF_MEMORY;
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->counters, 3 * sizeof(DevCounters));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->exposure, sizeof(float));
  if (e == cudaSuccess) e = cudaMallocHost(&ctx->h_ctl, kCtlWords * sizeof(uint32_t));
  if (e != cudaSuccess) {
    lgpu_destroy(ctx);
    return e == cudaErrorMemoryAllocation ? LGPU_ERR_OUT_OF_MEMORY : LGPU_ERR_CUDA;
  }
  *out = ctx;
  return LGPU_OK;
}

void lgpu_destroy(lgpu_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->release_scene();
  ctx->out.release();
  ctx->w_arena.release();
  ctx->jobs.release();
  ctx->job_items.release();
  ctx->job_pixels.release();
  ctx->batch_out.release();
  ctx->adj_buf.release();
  if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
  ctx->rays.release();
  ctx->hits.release();
  ctx->trace_arena.release();
  ctx->trace_tmax.release();
  ctx->trace_skip.release();
  ctx->trace_any.release();
  ctx->raw.release();
  ctx->layout_err.release();
  ctx->probes.release();
  ctx->probe_out.release();
  ctx->partials.release();
  ctx->tm_in.release();
  ctx->tm_out.release();
  ctx->tm_24.release();
  if (ctx->counters) cudaFree(ctx->counters);
  if (ctx->exposure) cudaFree(ctx->exposure);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  ctx->graph.release();
  for (auto& k : ctx->launch.ev)
    for (auto& s : k)
      for (cudaEvent_t ev : s)
        if (ev) cudaEventDestroy(ev);
  if (ctx->side) {
    cudaStreamSynchronize(ctx->side);
    cudaStreamDestroy(ctx->side);
  }
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* lgpu_last_error(const lgpu_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int lgpu_upload_scene(lgpu_ctx* ctx, const lgpu_scene* scene) {
  if (!ctx || !scene) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument");
  return lgpu_upload_scenes(ctx, &scene, 1);
}

int lgpu_upload_scenes(lgpu_ctx* ctx, const lgpu_scene* const* scenes, uint32_t n) {
  if (!ctx || !scenes || n == 0) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument or no scene");
  if (int r = bind_device(ctx)) return r;
  for (uint32_t k = 0; k < n; k++) {
    if (!scenes[k]) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null scene " + std::to_string(k));
    if (scenes[k]->spec.hero_k != scenes[0]->spec.hero_k)
      return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "all scenes of a table need the same hero-wavelength count");
  }
  cudaStreamSynchronize(ctx->stream);
  // slots keep their device allocations for the next upload
  for (size_t k = n; k < ctx->slots.size(); k++) ctx->slots[k].release();
  ctx->slots.resize(n);
  ctx->has_scene = false;
  ctx->stats.max_stack = 0;
  uint64_t total = 0;
  for (uint32_t k = 0; k < n; k++) {
    int const rc = upload_slot(ctx, ctx->slots[k], *scenes[k]);
    if (rc != LGPU_OK) {
      ctx->release_scene();
      return rc;
    }
    total += ctx->slots[k].bytes;
  }
  ctx->S = ctx->slots[0].S;
  ctx->stats.upload_bytes = total;
  ctx->has_scene = true;
  return LGPU_OK;
}

int lgpu_update_materials(lgpu_ctx* ctx, const lgpu_scene* scene) {
  if (!ctx || !scene) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (int r = bind_device(ctx)) return r;
  if (!ctx->has_scene) return fail(ctx, LGPU_ERR_NO_SCENE, "no scene uploaded");
  SceneSlot& sl = ctx->slots[0];
  if (scene->n_materials != sl.S.n_materials || size_t(scene->n_spectra) * scene->spec.n_bins != sl.spectra.n ||
      scene->spec.n_bins != sl.S.n_bins || (scene->n_spectra && !scene->spectra))
    return fail(ctx, LGPU_ERR_INVALID_ARGUMENT,
                "the material and spectrum counts must match the uploaded scene");
  std::vector<DevMaterial> mats;
  std::string err;
  if (int rc = make_materials(*scene, mats, err)) return fail(ctx, rc, err);
  cudaStream_t const st = ctx->stream;
  cudaError_t e = cudaSuccess;
  if (!mats.empty())
    e = cudaMemcpyAsync(sl.mats.ptr, mats.data(), mats.size() * sizeof(DevMaterial), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && sl.spectra.n)
    e = cudaMemcpyAsync(sl.spectra.ptr, scene->spectra, sl.spectra.n * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "material update");
  return LGPU_OK;
}

int lgpu_render_device(lgpu_ctx* ctx, const lgpu_render_params* params, float* d_out, void* stream) {
  if (!ctx || !d_out) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (int r = bind_device(ctx)) return r;
  cudaStream_t const user = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  cudaError_t e = fork_from(ctx, user);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "render");
  int const rc = render_impl(ctx, params, d_out, ctx->stream);
  if (rc != LGPU_OK) return rc;
  e = join_to(ctx, user);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "render");
  return collect(ctx, "render", timing_requested(params));
}

int lgpu_render(lgpu_ctx* ctx, const lgpu_render_params* params, float* out_linrgb) {
  if (!ctx || !out_linrgb) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (int r = bind_device(ctx)) return r;
  if (!ctx->has_scene) return fail(ctx, LGPU_ERR_NO_SCENE, "no scene uploaded");
  size_t const n = size_t(ctx->S.cam.width) * ctx->S.cam.height * 3;
  // an FP64 film writes doubles: twice the floats
  size_t const nf = (params && (params->flags & LGPU_FLAG_FP64_FILM)) ? 2 * n : n;
  cudaError_t e = ensure(ctx->out, nf);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "output buffer");
  int const rc = render_impl(ctx, params, ctx->out.ptr, ctx->stream);
  if (rc != LGPU_OK) return rc;
  e = cudaMemcpyAsync(out_linrgb, ctx->out.ptr, nf * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "render readback");
  return collect(ctx, "render", timing_requested(params));
}

int lgpu_render_batch_device(lgpu_ctx* ctx, const lgpu_job* jobs, uint32_t n, void* stream) {
  if (!ctx || !jobs || n == 0) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument or no job");
  if (int r = bind_device(ctx)) return r;
  cudaStream_t const user = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  std::vector<float*> outs(n);
  for (uint32_t k = 0; k < n; k++) outs[k] = jobs[k].out;
  cudaError_t e = fork_from(ctx, user);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "render batch");
  int const rc = batch_impl(ctx, jobs, n, outs.data(), ctx->stream);
  if (rc != LGPU_OK) return rc;
  e = join_to(ctx, user);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "render batch");
  return collect(ctx, "render batch", batch_timing(jobs, n));
}

int lgpu_render_batch(lgpu_ctx* ctx, const lgpu_job* jobs, uint32_t n) {
  if (!ctx || !jobs || n == 0) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument or no job");
  if (int r = bind_device(ctx)) return r;
  if (!ctx->has_scene) return fail(ctx, LGPU_ERR_NO_SCENE, "no scene uploaded");
  std::vector<size_t> off(n + 1, 0);
  for (uint32_t k = 0; k < n; k++) {
    if (jobs[k].scene >= ctx->slots.size())
      return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "job " + std::to_string(k) + ": no such scene");
    if (!jobs[k].out) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "job " + std::to_string(k) + ": null output");
    const lgpu_camera& c = ctx->slots[jobs[k].scene].S.cam;
    off[k + 1] = off[k] + size_t(c.width) * c.height * 3;
  }
  cudaError_t e = ensure(ctx->batch_out, off[n]);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch output buffer");
  std::vector<float*> outs(n);
  for (uint32_t k = 0; k < n; k++) outs[k] = ctx->batch_out.ptr + off[k];
  int const rc = batch_impl(ctx, jobs, n, outs.data(), ctx->stream);
  if (rc != LGPU_OK) return rc;
  // each job's rectangle of its frame (tile jobs may share a host output)
  for (uint32_t k = 0; k < n && e == cudaSuccess; k++) {
    const lgpu_camera& c = ctx->slots[jobs[k].scene].S.cam;
    uint32_t x0, r0, tw, th;
    job_rect(jobs[k], c, x0, r0, tw, th);
    size_t const pitch = size_t(c.width) * 3 * sizeof(float);
    size_t const first = (size_t(c.height - r0 - th) * c.width + x0) * 3;
    e = cudaMemcpy2DAsync(jobs[k].out + first, pitch, outs[k] + first, pitch, size_t(tw) * 3 * sizeof(float), th,
                          cudaMemcpyDeviceToHost, ctx->stream);
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch readback");
  return collect(ctx, "render batch", batch_timing(jobs, n));
}

int lgpu_adjoint_device(lgpu_ctx* ctx, const lgpu_render_params* params, const float* d_dloss_dimage,
                        float* d_grad_spectra, float* d_grad_materials, float* d_out_linrgb, void* stream) {
  if (!ctx || !params || !d_dloss_dimage || !d_grad_spectra || !d_grad_materials)
    return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (int r = bind_device(ctx)) return r;
  cudaStream_t const user = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  cudaError_t e = fork_from(ctx, user);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint");
  int const rc = adjoint_impl(ctx, params, d_dloss_dimage, d_grad_spectra, d_grad_materials, d_out_linrgb,
                              ctx->stream);
  if (rc != LGPU_OK) return rc;
  e = join_to(ctx, user);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint");
  return collect(ctx, "adjoint", (params->flags & LGPU_FLAG_KERNEL_TIMING) != 0);
}

int lgpu_adjoint(lgpu_ctx* ctx, const lgpu_render_params* params, const float* dloss_dimage, float* grad_spectra,
                 float* grad_materials, float* out_linrgb) {
  if (!ctx || !params || !dloss_dimage || !grad_spectra || !grad_materials)
    return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (int r = bind_device(ctx)) return r;
  if (!ctx->has_scene) return fail(ctx, LGPU_ERR_NO_SCENE, "no scene uploaded");
  size_t const npx = size_t(ctx->S.cam.width) * ctx->S.cam.height * 3;
  size_t const n_spec = ctx->slots[0].spectra.n;
  size_t const n_mat = 4 * size_t(ctx->S.n_materials);
  // one device buffer: dLoss/dimage, image, spectral and material gradients
  cudaError_t e = ensure(ctx->adj_buf, 2 * npx + n_spec + n_mat);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint buffers");
  float* const d_dimg = ctx->adj_buf.ptr;
  float* const d_img = d_dimg + npx;
  float* const d_gs = d_img + npx;
  float* const d_gm = d_gs + n_spec;
  cudaStream_t const st = ctx->stream;
  e = cudaMemcpyAsync(d_dimg, dloss_dimage, npx * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint upload");
  int const rc = adjoint_impl(ctx, params, d_dimg, d_gs, d_gm, out_linrgb ? d_img : nullptr, st);
  if (rc != LGPU_OK) return rc;
  e = cudaMemcpyAsync(grad_spectra, d_gs, n_spec * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(grad_materials, d_gm, n_mat * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && out_linrgb)
    e = cudaMemcpyAsync(out_linrgb, d_img, npx * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint readback");
  return collect(ctx, "adjoint", (params->flags & LGPU_FLAG_KERNEL_TIMING) != 0);
}

int lgpu_get_wave_config(const lgpu_ctx* ctx, lgpu_wave_config* out) {
  if (!ctx || !out) return LGPU_ERR_INVALID_ARGUMENT;
  out->queue_cap = ctx->cfg.queue_cap;
  out->shade_block = ctx->cfg.shade_block;
  out->trace_per_sm = ctx->cfg.trace_per_sm;
  out->graphs = ctx->cfg.graphs;
  out->mega_items = ctx->cfg.mega_items;
  return LGPU_OK;
}

int lgpu_set_wave_config(lgpu_ctx* ctx, const lgpu_wave_config* c) {
  if (!ctx || !c) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (c->queue_cap < 1024 || c->queue_cap > (1u << 24))
    return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "queue_cap must be in [1024, 2^24]");
  if (c->shade_block < 32 || c->shade_block > kMaxShadeBlock || c->shade_block % 32)
    return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "shade_block must be a multiple of 32 up to 256");
  ctx->cfg.queue_cap = c->queue_cap;
  ctx->cfg.shade_block = c->shade_block;
  ctx->cfg.trace_per_sm = c->trace_per_sm;
  ctx->cfg.graphs = c->graphs ? 1 : 0;
  ctx->cfg.mega_items = c->mega_items;
  return LGPU_OK;
}

int lgpu_autotune_batch(lgpu_ctx* ctx, const lgpu_job* jobs, uint32_t n, uint32_t spp_divisor,
                        lgpu_wave_config* out) {
  if (!ctx || !jobs || n == 0) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument or no job");
  if (int r = bind_device(ctx)) return r;
  if (!ctx->has_scene) return fail(ctx, LGPU_ERR_NO_SCENE, "no scene uploaded");
  uint32_t const div = spp_divisor ? spp_divisor : 1;
  std::vector<lgpu_job> sample(jobs, jobs + n);
  std::vector<size_t> off(n + 1, 0);
  for (uint32_t k = 0; k < n; k++) {
    if (sample[k].scene >= ctx->slots.size())
      return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "job " + std::to_string(k) + ": no such scene");
    sample[k].params.spp = std::max(1u, sample[k].params.spp / div);
    sample[k].params.flags &= ~uint32_t(LGPU_FLAG_KERNEL_TIMING);
    const lgpu_camera& c = ctx->slots[sample[k].scene].S.cam;
    off[k + 1] = off[k] + size_t(c.width) * c.height * 3;
  }
  cudaError_t e = ensure(ctx->batch_out, off[n]);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "autotune output buffer");
  std::vector<float*> outs(n);
  for (uint32_t k = 0; k < n; k++) outs[k] = ctx->batch_out.ptr + off[k];
  // device time of the sample batch under the current configuration
  auto measure = [&](double& ms) -> int {
    float best = 1e30f;
    for (int rep = 0; rep < 2; rep++) {
      cudaEvent_t e0 = ctx->ev0, e1 = ctx->ev1;
      cudaError_t ce = cudaEventRecord(e0, ctx->stream);
      if (ce != cudaSuccess) return cuda_fail(ctx, ce, "autotune");
      int const rc = batch_impl(ctx, sample.data(), n, outs.data(), ctx->stream);
      if (rc != LGPU_OK) return rc;
      ce = cudaEventRecord(e1, ctx->stream);
      if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
      float t = 0.f;
      if (ce == cudaSuccess) ce = cudaEventElapsedTime(&t, e0, e1);
      if (ce != cudaSuccess) return cuda_fail(ctx, ce, "autotune");
      best = std::min(best, t);
    }
    ms = best;
    return LGPU_OK;
  };
  WaveConfig const saved = ctx->cfg;
  WaveConfig best = ctx->cfg;
  double best_ms = 0.0;
  if (int rc = measure(best_ms)) {
    ctx->cfg = saved;
    return rc;
  }
  // coordinate descent over the knobs, each from the best so far
  auto try_dim = [&](auto set, std::initializer_list<uint64_t> values) -> int {
    WaveConfig const base = best;
    for (uint64_t v : values) {
      ctx->cfg = base;
      set(ctx->cfg, v);
      if (std::memcmp(&ctx->cfg, &base, sizeof(WaveConfig)) == 0) continue;
      double ms = 0.0;
      if (int rc = measure(ms)) return rc;
      if (ms < best_ms) {
        best_ms = ms;
        best = ctx->cfg;
      }
    }
    return LGPU_OK;
  };
  int rc = try_dim([](WaveConfig& c, uint64_t v) { c.queue_cap = uint32_t(v); },
                   {1u << 20, 1u << 22, 1u << 23, 1u << 24});
  if (!rc) rc = try_dim([](WaveConfig& c, uint64_t v) { c.shade_block = uint32_t(v); }, {64, 128, 256});
  if (!rc) rc = try_dim([](WaveConfig& c, uint64_t v) { c.trace_per_sm = uint32_t(v); }, {0, 4, 5});
  if (!rc) rc = try_dim([](WaveConfig& c, uint64_t v) { c.graphs = uint32_t(v); }, {0, 1});
  if (!rc) rc = try_dim([](WaveConfig& c, uint64_t v) { c.mega_items = v; }, {0, 1u << 14, 1u << 16});
  if (rc) {
    ctx->cfg = saved;
    return rc;
  }
  ctx->cfg = best;
  ctx->stats.last_kernel_ms = best_ms;
  if (out) lgpu_get_wave_config(ctx, out);
  return LGPU_OK;
}

}  // extern "C"

namespace {

// lgpu_trace_closest / lgpu_trace_any: the rays in chunks of at most
// kTraceChunk through the render's traversal kernels (lgpu_trace.cu).
constexpr uint64_t kTraceChunk = uint64_t(1) << 22;

int trace_impl(lgpu_ctx* ctx, const float* rays, const float* tmax, const uint32_t* skip, uint64_t n,
               uint32_t flags, lgpu_hit* out, uint8_t* out_any) {
  bool const any = out_any != nullptr;
  if (int r = bind_device(ctx)) return r;
  if (!ctx->has_scene) return fail(ctx, LGPU_ERR_NO_SCENE, "no scene uploaded");
  if (n == 0) return LGPU_OK;
  uint32_t const cap = uint32_t(n < kTraceChunk ? n : kTraceChunk);
  WaveState w{};
  size_t const bytes = trace_wave_layout(nullptr, cap, w);
  cudaError_t e = ensure(ctx->trace_arena, bytes);
  if (e == cudaSuccess) e = ensure(ctx->rays, 6 * size_t(cap));
  if (e == cudaSuccess && !any) e = ensure(ctx->hits, cap);
  if (e == cudaSuccess && any) e = ensure(ctx->trace_tmax, cap);
  if (e == cudaSuccess && any) e = ensure(ctx->trace_skip, cap);
  if (e == cudaSuccess && any) e = ensure(ctx->trace_any, cap);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "ray buffers");
  trace_wave_layout(ctx->trace_arena.ptr, cap, w);
  cudaStream_t const st = ctx->stream;
  e = cudaMemsetAsync(ctx->counters, 0, 3 * sizeof(DevCounters), st);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, st);
  ctx->launch.reset(false);
  uint64_t const chunks = (n + cap - 1) / cap;
  // setup, load, store + the traversal (persistent + fallback, or linear)
  ctx->launch.total = chunks * (any ? 4 : ((flags & LGPU_FLAG_REFERENCE_ORDER) || ctx->S.n_objects <= 4 ? 4 : 5));
  for (uint64_t c0 = 0; c0 < n && e == cudaSuccess; c0 += cap) {
    uint32_t const m = uint32_t(n - c0 < cap ? n - c0 : cap);
    e = cudaMemcpyAsync(ctx->rays.ptr, rays + 6 * c0, 6 * size_t(m) * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && any)
      e = cudaMemcpyAsync(ctx->trace_tmax.ptr, tmax + c0, m * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && any)
      e = cudaMemcpyAsync(ctx->trace_skip.ptr, skip + c0, m * sizeof(uint32_t), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = launch_trace_chunk(ctx->S, w, ctx->rays.ptr, ctx->trace_tmax.ptr, ctx->trace_skip.ptr, m, any, flags,
                             ctx->hits.ptr, ctx->trace_any.ptr, ctx->cfg, ctx->counters, st);
    if (e == cudaSuccess && !any)
      e = cudaMemcpyAsync(out + c0, ctx->hits.ptr, m * sizeof(lgpu_hit), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && any)
      e = cudaMemcpyAsync(out_any + c0, ctx->trace_any.ptr, m, cudaMemcpyDeviceToHost, st);
    // the staging buffers are reused by the next chunk
    if (e == cudaSuccess && c0 + cap < n) e = cudaStreamSynchronize(st);
  }
  if (e == cudaSuccess) e = cudaEventRecord(ctx->ev1, st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "trace");
  return collect(ctx, "trace");
}

}  // namespace

extern "C" {

int lgpu_trace_closest(lgpu_ctx* ctx, const float* rays, uint64_t n, uint32_t flags, lgpu_hit* out) {
  if (!ctx || (n && (!rays || !out))) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument");
  return trace_impl(ctx, rays, nullptr, nullptr, n, flags, out, nullptr);
}

int lgpu_trace_any(lgpu_ctx* ctx, const float* rays, const float* tmax, const uint32_t* skip, uint64_t n,
                   uint32_t flags, uint8_t* out_hit) {
  if (!ctx || (n && (!rays || !tmax || !skip || !out_hit)))
    return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument");
  return trace_impl(ctx, rays, tmax, skip, n, flags, nullptr, out_hit);
}

int lgpu_probe_shading(lgpu_ctx* ctx, const lgpu_probe* queries, uint64_t n, lgpu_probe_result* out) {
  if (!ctx || (n && (!queries || !out))) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (int r = bind_device(ctx)) return r;
  if (!ctx->has_scene) return fail(ctx, LGPU_ERR_NO_SCENE, "no scene uploaded");
  if (n == 0) return LGPU_OK;
  const DevScene& S = ctx->S;
  uint64_t const n_spectra = S.n_bins ? ctx->slots[0].spectra.n / S.n_bins : 0;
  for (uint64_t q = 0; q < n; q++) {
    lgpu_probe const& Q = queries[q];
    uint64_t bound = 0;
    switch (Q.op) {
      case LGPU_PROBE_BXDF:
      case LGPU_PROBE_PROB_MATERIAL:
      case LGPU_PROBE_SAMPLE_MATERIAL: bound = S.n_materials; break;
      case LGPU_PROBE_SAMPLE_LIGHT:
      case LGPU_PROBE_PROB_LIGHT: bound = S.n_lights; break;
      case LGPU_PROBE_SPECTRUM: bound = n_spectra; break;
      default:
        return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "probe " + std::to_string(q) + ": unknown op");
    }
    if (Q.index >= bound)
      return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "probe " + std::to_string(q) + ": index out of range");
  }
  cudaError_t e = ensure(ctx->probes, n);
  if (e == cudaSuccess) e = ensure(ctx->probe_out, n);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "probe buffers");
  cudaStream_t const st = ctx->stream;
  e = cudaMemcpyAsync(ctx->probes.ptr, queries, n * sizeof(lgpu_probe), cudaMemcpyHostToDevice, st);
  ctx->stats.launches = 1;
  if (e == cudaSuccess) e = launch_probe(S, ctx->probes.ptr, n, ctx->probe_out.ptr, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, ctx->probe_out.ptr, n * sizeof(lgpu_probe_result), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "probe");
  return LGPU_OK;
}

int lgpu_tonemap(lgpu_ctx* ctx, const float* linrgb, uint64_t w, uint64_t h, float y_mid,
                 float* out_tonemapped, uint8_t* out_rgb24) {
  if (!ctx || !linrgb) return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument");
  if (int r = bind_device(ctx)) return r;
  if (w == 0 || h == 0) return LGPU_OK;
  // 3*w*h elements must not wrap around in the sizes below
  if (w > (uint64_t(1) << 40) || h > (uint64_t(1) << 40) / w)
    return fail(ctx, LGPU_ERR_TOO_LARGE, "tone map: w*h is beyond 2^40 pixels");
  uint64_t const n = w * h;
  cudaStream_t const st = ctx->stream;
  uint32_t const nb = tonemap_partials_needed(n);
  cudaError_t e = ensure(ctx->partials, nb);
  if (e == cudaSuccess) e = ensure(ctx->tm_in, 3 * n);
  if (e == cudaSuccess && out_tonemapped) e = ensure(ctx->tm_out, 3 * n);
  if (e == cudaSuccess && out_rgb24) e = ensure(ctx->tm_24, 3 * n);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tone-map buffers");
  e = cudaMemcpyAsync(ctx->tm_in.ptr, linrgb, 3 * n * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = launch_tonemap(ctx->tm_in.ptr, n, y_mid, ctx->partials.ptr, nb, ctx->exposure,
                       out_tonemapped ? ctx->tm_out.ptr : nullptr, out_rgb24 ? ctx->tm_24.ptr : nullptr, st);
  if (e == cudaSuccess && out_tonemapped)
    e = cudaMemcpyAsync(out_tonemapped, ctx->tm_out.ptr, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && out_rgb24)
    e = cudaMemcpyAsync(out_rgb24, ctx->tm_24.ptr, 3 * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "tone map");
  return LGPU_OK;
}

int lgpu_get_stats(const lgpu_ctx* ctx, lgpu_stats* out) {
  if (!ctx || !out) return LGPU_ERR_INVALID_ARGUMENT;
  *out = ctx->stats;
  return LGPU_OK;
}

int lgpu_build_bvh_device(lgpu_ctx* ctx, const float* V, uint32_t n_positions, const uint32_t* F,
                          uint32_t f_stride, uint32_t n_faces, uint32_t* nodes, uint32_t* n_nodes, float* bbs,
                          uint32_t* n_bbs, uint32_t* prim_idxs, uint32_t* n_prim_idxs) {
  if (!ctx) return LGPU_ERR_INVALID_ARGUMENT;
  if (!V || !F || f_stride < 3 || n_faces == 0 || !n_nodes || !n_bbs || !n_prim_idxs)
    return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "null argument, f_stride < 3 or no faces");
  for (uint32_t f = 0; f < n_faces; f++)
    for (int k = 0; k < 3; k++)
      if (F[size_t(f) * f_stride + k] >= n_positions)
        return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "face " + std::to_string(f) + ": vertex index out of range");
  // the reduction that reproduces the host's nl::min / nl::max folds
  // assumes ordered values
  for (size_t i = 0; i < 3 * size_t(n_positions); i++)
    if (!std::isfinite(V[i]))
      return fail(ctx, LGPU_ERR_INVALID_ARGUMENT, "vertex " + std::to_string(i / 3) + " is not finite");
  if (int r = bind_device(ctx)) return r;
  RefBvh B;
  cudaError_t e;
  try {
    e = build_bvh_device(V, n_positions, F, f_stride, n_faces, B, ctx->stream);
  } catch (const std::bad_alloc&) {
    return fail(ctx, LGPU_ERR_OUT_OF_MEMORY, "host memory for the BVH");
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "device BVH build");
  *n_nodes = B.n_nodes;
  *n_bbs = uint32_t(B.bbs.size() / 48);
  *n_prim_idxs = uint32_t(B.prim_idxs.size());
  if (nodes) std::memcpy(nodes, B.nodes.data(), B.nodes.size() * sizeof(uint32_t));
  if (bbs) std::memcpy(bbs, B.bbs.data(), B.bbs.size() * sizeof(float));
  if (prim_idxs) std::memcpy(prim_idxs, B.prim_idxs.data(), B.prim_idxs.size() * sizeof(uint32_t));
  return LGPU_OK;
}

int lgpu_build_traversal_bvh(const float* V, uint32_t n_positions, const uint32_t* F, uint32_t f_stride,
                             uint32_t n_faces, uint32_t* nodes, uint32_t* n_nodes, float* bbs, uint32_t* n_bbs,
                             uint32_t* prim_idxs, uint32_t* n_prim_idxs) {
  if (!V || !F || f_stride < 3 || n_faces == 0 || !n_nodes || !n_bbs || !n_prim_idxs)
    return LGPU_ERR_INVALID_ARGUMENT;
  for (uint32_t f = 0; f < n_faces; f++)
    for (int k = 0; k < 3; k++)
      if (F[size_t(f) * f_stride + k] >= n_positions) return LGPU_ERR_INVALID_ARGUMENT;
  try {
    std::vector<PrimBox> boxes;
    std::vector<float> cents;
    triangle_prims(V, F, f_stride, n_faces, boxes, cents);
    for (const PrimBox& b : boxes)
      for (int k = 0; k < 3; k++)
        if (!std::isfinite(b.inf[k]) || !std::isfinite(b.sup[k])) return LGPU_ERR_INVALID_ARGUMENT;
    for (float c : cents)
      if (!std::isfinite(c)) return LGPU_ERR_INVALID_ARGUMENT;
    RefBvh B;
    build_sah_bvh(n_faces, boxes.data(), cents.data(), B, 2);
    *n_nodes = B.n_nodes;
    *n_bbs = uint32_t(B.bbs.size() / 48);
    *n_prim_idxs = uint32_t(B.prim_idxs.size());
    if (nodes) std::memcpy(nodes, B.nodes.data(), B.nodes.size() * sizeof(uint32_t));
    if (bbs) std::memcpy(bbs, B.bbs.data(), B.bbs.size() * sizeof(float));
    if (prim_idxs) std::memcpy(prim_idxs, B.prim_idxs.data(), B.prim_idxs.size() * sizeof(uint32_t));
  } catch (const std::bad_alloc&) {
    return LGPU_ERR_OUT_OF_MEMORY;
  } catch (const std::exception&) {
    return LGPU_ERR_OUT_OF_MEMORY;  // no threads for the build
  }
  return LGPU_OK;
}

int lgpu_build_bvh(const float* V, uint32_t n_positions, const uint32_t* F, uint32_t f_stride,
                   uint32_t n_faces, uint32_t* nodes, uint32_t* n_nodes, float* bbs, uint32_t* n_bbs,
                   uint32_t* prim_idxs, uint32_t* n_prim_idxs) {
  if (!V || !F || f_stride < 3 || n_faces == 0 || !n_nodes || !n_bbs || !n_prim_idxs)
    return LGPU_ERR_INVALID_ARGUMENT;
  for (uint32_t f = 0; f < n_faces; f++)
    for (int k = 0; k < 3; k++)
      if (F[size_t(f) * f_stride + k] >= n_positions) return LGPU_ERR_INVALID_ARGUMENT;
  try {
    std::vector<PrimBox> boxes;
    std::vector<float> cents;
    triangle_prims(V, F, f_stride, n_faces, boxes, cents);
    RefBvh B;
    build_ref_bvh(n_faces, boxes.data(), cents.data(), B);
    *n_nodes = B.n_nodes;
    *n_bbs = uint32_t(B.bbs.size() / 48);
    *n_prim_idxs = uint32_t(B.prim_idxs.size());
    if (nodes) std::memcpy(nodes, B.nodes.data(), B.nodes.size() * sizeof(uint32_t));
    if (bbs) std::memcpy(bbs, B.bbs.data(), B.bbs.size() * sizeof(float));
    if (prim_idxs) std::memcpy(prim_idxs, B.prim_idxs.data(), B.prim_idxs.size() * sizeof(uint32_t));
  } catch (const std::bad_alloc&) {
    return LGPU_ERR_OUT_OF_MEMORY;
  }
  return LGPU_OK;
}

}  // extern "C"
