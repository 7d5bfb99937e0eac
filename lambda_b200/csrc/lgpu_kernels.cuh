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

// Device buffers of the wavefront renderer (lgpu_wave.cuh), per-path state
// in structure-of-arrays layout; the context owns them.
struct WaveState {
  uint32_t cap;      // path slots
  uint32_t npix;     // pixels of the frame
  uint32_t n_samples;  // samples per pixel in this wave (cap >= npix*n_samples)
  float* ray;        // 6*cap (ox, oy, oz, dx, dy, dz), field-major
  uint64_t* rng;     // cap
  float* hero;       // cap
  uint32_t* depth;   // cap
  float* beta;       // K*cap
  float* acc;        // K*cap
  float* hit;        // 9*cap (z, obj, face, b0, b1, b2, plx, ply, plz)
  uint32_t* q_in;    // active path slots
  uint32_t* q_out;
  uint32_t* n_in;    // device counts
  uint32_t* n_out;
  float* sray;       // 8*cap (ox, oy, oz, dx, dy, dz, tmax, skip)
  uint32_t* s_path;  // cap
  float* s_contrib;  // K*cap
  uint32_t* n_shadow;
  uint32_t* fetch;     // 2 work counters of the persistent trace kernels
  uint32_t* fb_queue;  // extension rays re-traced in the reference's object order
  uint32_t* n_fb;
  // streaming: a slot whose path ends is refilled with the next
  // (sample, pixel) of the frame
  uint32_t* pix;        // cap: pixel of the slot's path
  uint32_t* samp;       // cap: sample index (relative to the chunk)
  uint32_t* free_list;  // cap
  uint32_t* fin_list;   // cap: slots whose path ended this iteration
  uint32_t* ctl;        // [0] free slots, [1] next work item, [2] ended paths,
                        // [3..6] plan of the next generate (new, first item,
                        // free-list top, queue position)
  uint32_t* h_ctl;      // pinned host copy of ctl[0..2] and the queue count
  float* sbuf;          // 3 * npix * n_samples: XYZ of every (sample, pixel)
  float* film;       // 3*npix XYZ
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
