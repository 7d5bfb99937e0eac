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

cudaError_t launch_render(const DevScene& S, const RenderArgs& a, float* d_out, DevCounters* d_cnt,
                          cudaStream_t st);
template <int K>
cudaError_t launch_render_k(const DevScene& S, const RenderArgs& a, float* d_out, DevCounters* d_cnt,
                            cudaStream_t st);

// Tone map: partial sums of log-luminance go to d_partials (n_partials
// doubles, at least tonemap_partials_needed(n)).
uint32_t tonemap_partials_needed(uint64_t n_pixels);
cudaError_t launch_tonemap(const float* d_rgb, uint64_t n_pixels, float y_mid, double* d_partials,
                           uint32_t n_partials, float* d_exposure, float* d_out_tm,
                           uint8_t* d_out24, cudaStream_t st);

}  // namespace lgpu
