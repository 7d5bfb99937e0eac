// lgpu_kernels.cuh — kernel entry points and their launch helpers.
#pragma once

#include <cuda_runtime.h>

#include "lgpu_scene.h"

namespace lgpu {

// Device-side counters written by the kernels (one per context).
struct DevCounters {
  unsigned long long rays;
  unsigned long long paths;
  unsigned long long nodes;  // wide-node child-box tests
  unsigned long long tris;   // triangle tests
  unsigned long long insts;  // object tests
  unsigned int flags;        // kTravOverflow, kTravLocalStack (lgpu_intersect.cuh)
  unsigned int nonfinite;    // paths whose radiance was NaN or infinite
  unsigned long long ordered; // rays re-traced in the reference's object order
};

// Path state of one queue of the wavefront renderer (lgpu_wave.cuh): path
// i of the queue at index i of every field, field-major.
struct PathBuf {
  float* ray;       // 6*cap (ox, oy, oz, dx, dy, dz)
  uint64_t* rng;    // cap
  float* hero;      // cap
  uint32_t* depth;  // cap
  uint32_t* item;   // cap: work item, relative to the first item of the chunk
  uint32_t* job;    // cap: job of the path (batched renders only)
  float* beta;      // K*cap
  float* acc;       // K*cap (path replay: the radiance still to come)
  float* gw;        // K*cap, path replay: dL/d(radiance) per hero wavelength
  uint32_t* sidx;   // cap: the path's shadow ray of the last iteration, or kNoShadow
};

// Counters of the wavefront renderer (WaveState::ctl).
constexpr int kCtlCountA = 0;    // queue lengths of the two PathBufs
constexpr int kCtlCountB = 1;
constexpr int kCtlShadow = 2;    // shadow rays
constexpr int kCtlFetch = 3;     // 2 work counters of the persistent trace kernels
constexpr int kCtlFallback = 5;  // rays re-traced in the reference's object order
constexpr int kCtlEnded = 6;     // ended paths
constexpr int kCtlNext = 7;      // next work item to start
constexpr int kCtlNew = 8;       // plan of the next generate: new paths,
constexpr int kCtlFirst = 9;     //   their first work item,
constexpr int kCtlPos = 10;      //   their first queue position
constexpr int kCtlListB = 11;    // queue entries that hit a Blinn material
constexpr int kCtlListT = 12;    //   and a thin-film one (shading lists)
constexpr int kCtlWords = 16;
constexpr uint32_t kNoShadow = 0xFFFFFFFFu;

// Device buffers of the wavefront renderer; the context owns them.
struct WaveState {
  uint32_t cap;        // queue capacity (paths in flight)
  uint32_t npix;       // pixels of the frame (of all frames of a batch)
  uint32_t n_samples;  // samples per pixel in one chunk of the frame
  uint64_t c0;         // first work item of the current chunk
  PathBuf in, out;     // current and next queue, swapped every iteration
  uint32_t* n_in;      // queue lengths (in ctl), swapped with the queues
  uint32_t* n_out;
  float* hit;          // 9*cap closest hits of `in` (z, obj, face, b0, b1, b2, plx, ply, plz)
  float* e_acc;        // K*cap: radiance of the paths ended this iteration
  float* e_hero;       // cap
  uint32_t* e_item;    // cap
  uint32_t* e_job;     // cap (batched renders only)
  float* sray;         // 8*cap shadow rays (ox, oy, oz, dx, dy, dz, tmax, skip)
  uint32_t* e_sidx;    // cap: the ended path's last shadow ray, or kNoShadow
  float* s_contrib;    // K*cap: contributions of this iteration's shadow rays
  float* s_prev;       // K*cap: those of the last iteration (swapped with s_contrib)
  uint8_t* s_vis;      // cap: 1 if the shadow ray reached its light
  uint32_t* s_job;     // cap (batched renders only)
  uint32_t* fb_queue;  // cap: `in` indices re-traced in the reference's object order
  uint32_t* shade_list;  // cap: `in` positions of the Blinn hits (from the front) and
                         // of the thin-film hits (from the back), for their shading launches
  uint32_t* ctl;       // kCtlWords counters
  uint32_t* h_ctl;     // pinned host copy of ctl
  float* sbuf;         // 3 per work item of a chunk: XYZ of every (sample, pixel)
  float* film;         // 3*npix XYZ
  double* film64;      // 3*npix XYZ in double (LGPU_FLAG_FP64_FILM), or nullptr
  // path replay (lgpu_adjoint): the primal pass records every path's
  // radiance and which of its shadow rays were unoccluded; the replay
  // pass reads them back
  float* ltot;         // K per work item of the chunk, or nullptr
  uint64_t* vis;       // per work item: bit v set = the shadow ray of vertex v reached its light
  uint32_t* s_item;    // cap: work item of each shadow ray
  uint32_t* s_depth;   // cap: its vertex
};

struct RenderArgs {
  uint32_t spp;
  uint32_t max_scatter;
  float sample_p;
  uint32_t flags;
  uint64_t seed;
  uint32_t spp_offset;
  uint32_t pixel_begin;  // first pixel (row-major, scene row order) of this launch
  uint32_t pixel_count;
  uint32_t stream_tag;   // high bits of the RNG stream id (job id)
};

// lgpu_probe_shading: one thread per query (lgpu_probe.cu)
cudaError_t launch_probe(const DevScene& S, const lgpu_probe* d_q, uint64_t n, lgpu_probe_result* d_out,
                         cudaStream_t st);

// Launch shape of the wavefront, chosen by the autotuner
// (lgpu_autotune_batch) or set by the caller (lgpu_set_wave_config).
// Largest block of the shading kernels, whose queue entries a block sorts
// by material together: 256 fills a warp with one material more often than
// 128 (shading -6 %; 512 is no faster)
constexpr uint32_t kMaxShadeBlock = 256;

struct WaveConfig {
  uint32_t queue_cap = 1u << 24;  // paths in flight
  uint32_t shade_block = 256;     // threads per block of the shading kernel (multiple of 32, <= 256)
  uint32_t trace_per_sm = 0;      // persistent trace blocks per SM (0: the occupancy limit)
  uint32_t graphs = 1;            // 1: bounce stages replayed from a captured CUDA graph
  uint64_t mega_items = 0;        // batches: jobs with fewer work items run the megakernel
};

// Instantiated CUDA graph of the bounce stages, updated in place while the
// stages keep their shape.
struct GraphCache {
  cudaGraphExec_t exec = nullptr;
  void release() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
  }
};

// Launch settings and bookkeeping of one render: the configuration, the
// graph cache, the number of kernel launches, and with `on` the device time
// of the wavefront's launches per kind (0 closest-hit traversal, 1 shadow
// traversal, 2 shading), from pairs of events recorded around each launch
// and read back after the stream synchronises (no graphs then).
struct WaveLaunch {
  static constexpr int kSlots = 16;
  WaveConfig cfg;
  GraphCache* graph = nullptr;
  unsigned long long graph_launches = 0;
  bool on = false;
  unsigned long long total = 0;  // kernel launches
  cudaEvent_t ev[3][kSlots][2] = {};
  int used[3] = {0, 0, 0};
  double ms[3] = {0, 0, 0};
  unsigned long long launches[3] = {0, 0, 0};
  void reset(bool timing) {
    on = timing;
    total = 0;
    graph_launches = 0;
    for (int k = 0; k < 3; k++) {
      used[k] = 0;
      ms[k] = 0.0;
      launches[k] = 0;
    }
  }
  void begin(int k, cudaStream_t st) {
    if (on) cudaEventRecord(ev[k][used[k]][0], st);
  }
  void end(int k, cudaStream_t st) {
    if (!on) return;
    cudaEventRecord(ev[k][used[k]][1], st);
    used[k]++;
    launches[k]++;
  }
  // after the stream has synchronised
  void harvest() {
    if (!on) return;
    for (int k = 0; k < 3; k++) {
      for (int i = 0; i < used[k]; i++) {
        float m = 0.f;
        if (cudaEventElapsedTime(&m, ev[k][i][0], ev[k][i][1]) == cudaSuccess) ms[k] += m;
      }
      used[k] = 0;
    }
  }
};

// One job of a batched render: a scene, its settings and its place in
// the batch.  Work items of the batch are numbered job after job; within a
// job, item q is sample q / npix of pixel q % npix.
struct DevJob {
  DevScene S;
  RenderArgs a;
  uint64_t item_base;  // first work item of the job
  uint32_t npix;       // pixels of its rectangle
  uint32_t pix_base;   // first pixel of the job in the batch film
  float* out;          // linear RGB of the whole frame, width*height*3, row 0 at the top
  uint32_t col0, row0, tile_w;  // rectangle: first column, first scene row, width
};

#ifdef __CUDACC__
// Job policies of the wavefront kernels.  OneJob (the plain renderer) keeps
// its scene and settings in kernel parameters; JobTable (a batch) reads
// them from a device table, and every path carries its job index.
struct OneJob {
  static constexpr bool kMulti = false;
  DevScene S;
  RenderArgs a;
  uint32_t npix;
  float* out;
  __device__ __forceinline__ const DevScene& scene(uint32_t) const { return S; }
  __device__ __forceinline__ const RenderArgs& args(uint32_t) const { return a; }
  __device__ __forceinline__ uint32_t job_of_item(uint64_t) const { return 0; }
  __device__ __forceinline__ uint32_t job_of_pixel(uint32_t) const { return 0; }
  __device__ __forceinline__ uint64_t item_base(uint32_t) const { return 0; }
  __device__ __forceinline__ uint32_t pix_base(uint32_t) const { return 0; }
  __device__ __forceinline__ uint32_t npix_of(uint32_t) const { return npix; }
  __device__ __forceinline__ float* out_of(uint32_t) const { return out; }
  // frame pixel (scene row-major) of the job's local pixel
  __device__ __forceinline__ uint32_t frame_pixel(uint32_t, uint32_t p) const { return p; }
};

struct JobTable {
  static constexpr bool kMulti = true;
  const DevJob* d;
  const uint64_t* item_bases;  // n + 1 entries, the last is the total
  const uint32_t* pix_bases;   // n + 1 entries
  uint32_t n;
  __device__ __forceinline__ const DevScene& scene(uint32_t j) const { return d[j].S; }
  __device__ __forceinline__ const RenderArgs& args(uint32_t j) const { return d[j].a; }
  // the job whose range holds item g / pixel gp (binary search)
  __device__ __forceinline__ uint32_t job_of_item(uint64_t g) const {
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
      uint32_t const mid = (lo + hi + 1) >> 1;
      if (item_bases[mid] <= g) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
  __device__ __forceinline__ uint32_t job_of_pixel(uint32_t gp) const {
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
      uint32_t const mid = (lo + hi + 1) >> 1;
      if (pix_bases[mid] <= gp) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
  __device__ __forceinline__ uint64_t item_base(uint32_t j) const { return item_bases[j]; }
  __device__ __forceinline__ uint32_t pix_base(uint32_t j) const { return pix_bases[j]; }
  __device__ __forceinline__ uint32_t npix_of(uint32_t j) const { return d[j].npix; }
  __device__ __forceinline__ float* out_of(uint32_t j) const { return d[j].out; }
  __device__ __forceinline__ uint32_t frame_pixel(uint32_t j, uint32_t p) const {
    const DevJob& jb = d[j];
    uint32_t const r = p / jb.tile_w;
    return (jb.row0 + r) * uint32_t(jb.S.cam.width) + jb.col0 + (p - r * jb.tile_w);
  }
};
#endif

// Ray-set queries through the render's traversal kernels (lgpu_trace.cu).
// trace_wave_layout lays out the queue fields they use for cap rays in one
// allocation at base (nullptr: only counts the bytes);
// launch_trace_chunk traces n <= cap rays: closest hits into d_hits
// (any = false) or, for shadow rays with their distance bound and object to
// skip, whether each is occluded into d_hit_any (any = true).
size_t trace_wave_layout(uint8_t* base, uint32_t cap, WaveState& ws);
cudaError_t launch_trace_chunk(const DevScene& S, WaveState& w, const float* d_rays, const float* d_tmax,
                               const uint32_t* d_skip, uint32_t n, bool any, uint32_t flags,
                               lgpu_hit* d_hits, uint8_t* d_hit_any, const WaveConfig& cfg, DevCounters* d_cnt,
                               cudaStream_t st);

// Batched render of the jobs of `table` (n jobs, n_items work items,
// n_pix pixels in all) with the wavefront kernels.
cudaError_t launch_batch(uint32_t hero_k, const DevJob* d_jobs, const uint64_t* d_item_bases,
                         const uint32_t* d_pix_bases, uint32_t n_jobs, uint64_t n_items,
                         uint64_t chunk_items, bool linear, WaveState* wave, DevCounters* d_cnt,
                         cudaStream_t st, WaveLaunch* run);
template <int K>
cudaError_t launch_batch_k(const DevJob* d_jobs, const uint64_t* d_item_bases, const uint32_t* d_pix_bases,
                           uint32_t n_jobs, uint64_t n_items, uint64_t chunk_items, bool linear,
                           WaveState* wave, DevCounters* d_cnt, cudaStream_t st, WaveLaunch* run);

// Renders with the wavefront kernels when wave != nullptr, else with the
// one-thread-per-pixel megakernel.  d_cnt points at 3 counter records:
// everything, and with run->on the closest-hit and shadow traversal apart.
template <int K>
cudaError_t launch_render_k(const DevScene& S, const RenderArgs& a, WaveState* wave, float* d_out,
                            DevCounters* d_cnt, cudaStream_t st, WaveLaunch* run);
cudaError_t launch_render(const DevScene& S, const RenderArgs& a, WaveState* wave, float* d_out,
                          DevCounters* d_cnt, cudaStream_t st, WaveLaunch* run);

// Path-replay adjoint (lgpu_adjoint.cuh): primal image (d_img, may be null)
// and gradients of the loss whose image gradient is dimg.
struct AdjointArgs {
  const float* dimg;  // dLoss/d(linear RGB), width*height*3, row 0 at the top
  float* g_spec;      // n_spectra * n_bins
  float* g_mat;       // n_materials * 4: thickness, alpha, 0, 0
};
cudaError_t launch_adjoint(uint32_t hero_k, const DevScene& S, const RenderArgs& a, WaveState* wave,
                           uint64_t chunk_items, float* d_img, const AdjointArgs& g, DevCounters* d_cnt,
                           cudaStream_t st, WaveLaunch* run);
template <int K>
cudaError_t launch_adjoint_k(const DevScene& S, const RenderArgs& a, WaveState* wave, uint64_t chunk_items,
                             float* d_img, const AdjointArgs& g, DevCounters* d_cnt, cudaStream_t st,
                             WaveLaunch* run);

// Tone map: partial sums of log-luminance go to d_partials (n_partials
// doubles, at least tonemap_partials_needed(n), which never exceeds
// kTonemapMaxPartials: the reduction is grid-strided over at most 8 blocks
// per SM of a 148-SM B200).
constexpr uint32_t kTonemapMaxPartials = 148 * 8;
uint32_t tonemap_partials_needed(uint64_t n_pixels);
cudaError_t launch_tonemap(const float* d_rgb, uint64_t n_pixels, float y_mid, double* d_partials,
                           uint32_t n_partials, float* d_exposure, float* d_out_tm,
                           uint8_t* d_out24, cudaStream_t st);

}  // namespace lgpu
