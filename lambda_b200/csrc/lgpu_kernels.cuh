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
  unsigned int flags;        // bit 0: traversal stack overflow
  unsigned int nonfinite;    // paths whose radiance was NaN or infinite
};

// Path state of one queue of the wavefront renderer (lgpu_wave.cuh): path
// i of the queue at index i of every field, field-major.
struct PathBuf {
  float* ray;       // 6*cap (ox, oy, oz, dx, dy, dz)
  uint64_t* rng;    // cap
  float* hero;      // cap
  uint32_t* depth;  // cap
  uint32_t* item;   // cap: work item (sample * npix + pixel, relative to the chunk)
  float* beta;      // K*cap
  float* acc;       // K*cap
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
constexpr int kCtlWords = 16;
constexpr uint32_t kEndedBit = 0x80000000u;

// Device buffers of the wavefront renderer; the context owns them.
struct WaveState {
  uint32_t cap;        // queue capacity (paths in flight)
  uint32_t npix;       // pixels of the frame
  uint32_t n_samples;  // samples per pixel in one chunk of the frame
  PathBuf in, out;     // current and next queue, swapped every iteration
  uint32_t* n_in;      // queue lengths (in ctl), swapped with the queues
  uint32_t* n_out;
  float* hit;          // 9*cap closest hits of `in` (z, obj, face, b0, b1, b2, plx, ply, plz)
  float* e_acc;        // K*cap: radiance of the paths ended this iteration
  float* e_hero;       // cap
  uint32_t* e_item;    // cap
  float* sray;         // 8*cap shadow rays (ox, oy, oz, dx, dy, dz, tmax, skip)
  uint32_t* s_target;  // cap: path of each shadow ray (`out` index, or ended index | kEndedBit)
  float* s_contrib;    // K*cap
  uint32_t* fb_queue;  // cap: `in` indices re-traced in the reference's object order
  uint32_t* ctl;       // kCtlWords counters
  uint32_t* h_ctl;     // pinned host copy of ctl
  float* sbuf;         // 3 * npix * n_samples: XYZ of every (sample, pixel)
  float* film;         // 3*npix XYZ
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

cudaError_t launch_trace(const DevScene& S, const float* d_rays, uint64_t n, uint32_t flags,
                         lgpu_hit* d_hits, DevCounters* d_cnt, cudaStream_t st);

// Launch bookkeeping of one render: the number of kernel launches, and
// with `on` the device time of the wavefront's launches per kind (0
// closest-hit traversal, 1 shadow traversal, 2 shading), from pairs of
// events recorded around each launch and read back after the stream
// synchronises.
struct KernelTimer {
  static constexpr int kSlots = 16;
  bool on = false;
  unsigned long long total = 0;  // kernel launches
  cudaEvent_t ev[3][kSlots][2] = {};
  int used[3] = {0, 0, 0};
  double ms[3] = {0, 0, 0};
  unsigned long long launches[3] = {0, 0, 0};
  void reset(bool timing) {
    on = timing;
    total = 0;
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

// Renders with the wavefront kernels when wave != nullptr, else with the
// one-thread-per-pixel megakernel.  d_cnt points at 3 counter records:
// everything, and with timer->on the closest-hit and shadow traversal apart.
template <int K>
cudaError_t launch_render_k(const DevScene& S, const RenderArgs& a, WaveState* wave, float* d_out,
                            DevCounters* d_cnt, cudaStream_t st, KernelTimer* timer);
cudaError_t launch_render(const DevScene& S, const RenderArgs& a, WaveState* wave, float* d_out,
                          DevCounters* d_cnt, cudaStream_t st, KernelTimer* timer);

// Samples per pixel in one wave for a frame of npix pixels: enough paths in
// flight to fill the GPU (about 2^21), never more than spp.
uint32_t wave_samples(uint32_t npix, uint32_t spp);

// XYZ film (3 floats per pixel, scene row order) / norm * delta ->
// linear BT.709 RGB in the reference's layout (row 0 at the top),
// src/renderer.cpp:52-56.
cudaError_t launch_finalize(const float* film, uint32_t npix, uint32_t W, uint32_t H, float norm,
                            float delta, float* out, cudaStream_t st);

// Tone map: partial sums of log-luminance go to d_partials (n_partials
// doubles, at least tonemap_partials_needed(n)).
uint32_t tonemap_partials_needed(uint64_t n_pixels);
cudaError_t launch_tonemap(const float* d_rgb, uint64_t n_pixels, float y_mid, double* d_partials,
                           uint32_t n_partials, float* d_exposure, float* d_out_tm,
                           uint8_t* d_out24, cudaStream_t st);

}  // namespace lgpu
