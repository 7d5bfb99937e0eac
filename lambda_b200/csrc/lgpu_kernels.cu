// lgpu_kernels.cu — closest-hit, render and tone-map kernels.
#include <float.h>
#include <stdint.h>

#include "lgpu_counters.cuh"
#include "lgpu_kernels.cuh"

namespace lgpu {

namespace {

// ---- tone map (src/renderer.cpp:149-176) -------------------------------------

constexpr int kTmThreads = 256;
constexpr uint32_t kTmMaxBlocks = kTonemapMaxPartials;

// log-average luminance: per-block sums of log(max(Y, ε)) in double
__global__ void __launch_bounds__(kTmThreads) tm_logsum_kernel(const float* __restrict__ rgb, uint64_t n,
                                                               double* __restrict__ partials) {
  double s = 0.0;
  for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
       p += uint64_t(gridDim.x) * blockDim.x) {
    float const Yl = 0.2126f * rgb[3 * p] + 0.7152f * rgb[3 * p + 1] + 0.0722f * rgb[3 * p + 2];
    float const y = Yl >= kEps ? Yl : kEps;
    s += double(logf(y));
  }
  __shared__ double red[kTmThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kTmThreads / 32; w++) t += red[w];
    partials[blockIdx.x] = t;
  }
}

__global__ void tm_exposure_kernel(const double* __restrict__ partials, uint32_t nb, uint64_t n, float y_mid,
                                   float* __restrict__ exposure) {
  __shared__ double red[32];
  double s = 0.0;
  for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) s += partials[b];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (uint32_t w = 0; w < (blockDim.x + 31) / 32; w++) t += red[w];
    float const ybar = expf(float(t / double(n)));
    exposure[0] = y_mid / ybar;
  }
}

// tonemapping::koiFilmic (cg.hpp:181-194)
__device__ __forceinline__ float koi_filmic(float L) {
  float const x = 10.f * L;
  return (x * (0.3f * x + 0.14f)) / (x * (0.3f * x + 2.8f) + 10.f);
}
// linRGB2sRGB (cg.hpp:149-154) and float2byte (numli.hpp:105-106)
__device__ __forceinline__ uint8_t srgb_byte(float c) {
  float const s = c > 0.0031308f ? 1.055f * powf(c, 1.f / 2.4f) - 0.055f : 12.92f * c;
  int v = int(255.f * s + 0.5f);
  v = v < 0 ? 0 : (v > 255 ? 255 : v);
  return uint8_t(v);
}

__global__ void __launch_bounds__(kTmThreads) tm_map_kernel(const float* __restrict__ rgb, uint64_t n,
                                                            const float* __restrict__ exposure,
                                                            float* __restrict__ out_tm,
                                                            uint8_t* __restrict__ out24) {
  float const e = exposure[0];
  for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < 3 * n;
       q += uint64_t(gridDim.x) * blockDim.x) {
    float const L = koi_filmic(e * rgb[q]);
    if (out_tm) out_tm[q] = L;
    if (out24) out24[q] = srgb_byte(L);
  }
}

}  // namespace

cudaError_t launch_render(const DevScene& S, const RenderArgs& a, WaveState* wave, float* d_out,
                          DevCounters* d_cnt, cudaStream_t st, WaveLaunch* run) {
  if (a.pixel_count == 0) return cudaSuccess;
  switch (S.hero_k) {
    case 4: return launch_render_k<4>(S, a, wave, d_out, d_cnt, st, run);
    case 8: return launch_render_k<8>(S, a, wave, d_out, d_cnt, st, run);
    case 16: return launch_render_k<16>(S, a, wave, d_out, d_cnt, st, run);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_batch(uint32_t hero_k, const DevJob* d_jobs, const uint64_t* d_item_bases,
                         const uint32_t* d_pix_bases, uint32_t n_jobs, uint64_t n_items,
                         uint64_t chunk_items, bool linear, WaveState* wave, DevCounters* d_cnt,
                         cudaStream_t st, WaveLaunch* run) {
  if (n_jobs == 0 || n_items == 0) return cudaSuccess;
  switch (hero_k) {
    case 4:
      return launch_batch_k<4>(d_jobs, d_item_bases, d_pix_bases, n_jobs, n_items, chunk_items, linear, wave,
                               d_cnt, st, run);
    case 8:
      return launch_batch_k<8>(d_jobs, d_item_bases, d_pix_bases, n_jobs, n_items, chunk_items, linear, wave,
                               d_cnt, st, run);
    case 16:
      return launch_batch_k<16>(d_jobs, d_item_bases, d_pix_bases, n_jobs, n_items, chunk_items, linear, wave,
                                d_cnt, st, run);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_adjoint(uint32_t hero_k, const DevScene& S, const RenderArgs& a, WaveState* wave,
                           uint64_t chunk_items, float* d_img, const AdjointArgs& g, DevCounters* d_cnt,
                           cudaStream_t st, WaveLaunch* run) {
  switch (hero_k) {
    case 4: return launch_adjoint_k<4>(S, a, wave, chunk_items, d_img, g, d_cnt, st, run);
    case 8: return launch_adjoint_k<8>(S, a, wave, chunk_items, d_img, g, d_cnt, st, run);
    case 16: return launch_adjoint_k<16>(S, a, wave, chunk_items, d_img, g, d_cnt, st, run);
  }
  return cudaErrorInvalidValue;
}

uint32_t tonemap_partials_needed(uint64_t n_pixels) {
  uint64_t const b = (n_pixels + kTmThreads - 1) / kTmThreads;
  return uint32_t(b < kTmMaxBlocks ? (b ? b : 1) : kTmMaxBlocks);
}

cudaError_t launch_tonemap(const float* d_rgb, uint64_t n_pixels, float y_mid, double* d_partials,
                           uint32_t n_partials, float* d_exposure, float* d_out_tm, uint8_t* d_out24,
                           cudaStream_t st) {
  uint32_t const nb = tonemap_partials_needed(n_pixels);
  if (n_partials < nb) return cudaErrorInvalidValue;
  tm_logsum_kernel<<<nb, kTmThreads, 0, st>>>(d_rgb, n_pixels, d_partials);
  tm_exposure_kernel<<<1, 1024, 0, st>>>(d_partials, nb, n_pixels, y_mid, d_exposure);
  uint64_t const mb = (3 * n_pixels + kTmThreads - 1) / kTmThreads;
  uint32_t const map_blocks = uint32_t(mb < kTmMaxBlocks ? (mb ? mb : 1) : kTmMaxBlocks);
  tm_map_kernel<<<map_blocks, kTmThreads, 0, st>>>(d_rgb, n_pixels, d_exposure, d_out_tm, d_out24);
  return cudaGetLastError();
}

}  // namespace lgpu
