// lgpu_noalloc.cu — lgpu_tonemap_noalloc: the tone map with its scratch in
// a file-scope device array, for callers that cannot allocate device memory
// when they call it (see include/lambda_gpu.h).
//
// The tone map's scratch is the per-block partial sums of log-luminance
// (at most kTonemapMaxPartials doubles for any image, the reduction is
// grid-strided) and the exposure (one float).  Both live in
// g_tonemap_scratch; host code gets its device address once per device with
// cudaGetSymbolAddress (the symbol itself is only a host-side stand-in) and
// passes that address to the same kernels lgpu_tonemap launches.
#include <cuda_runtime.h>

#include <mutex>

#include "lambda_gpu.h"
#include "lgpu_kernels.cuh"

namespace {

constexpr uint32_t kPartials = lgpu::kTonemapMaxPartials;
constexpr size_t kScratchDoubles = LGPU_NOALLOC_SCRATCH_BYTES / sizeof(double);
static_assert(kScratchDoubles >= kPartials + 1, "partials + the exposure slot");

static __device__ __align__(256) double g_tonemap_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_tonemap_scratch on the current device, looked up once
// per device with that device current.  The address belongs to the device's
// primary context (the runtime's); it stays valid until that context is
// destroyed (cudaDeviceReset), after which this cache would be stale.
int scratch_address(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return LGPU_ERR_NO_DEVICE;
  if (dev < 0 || dev >= kMaxDevices) return LGPU_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    double* p = nullptr;
    cudaError_t const e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_tonemap_scratch);
    if (e != cudaSuccess || !p) return LGPU_ERR_CUDA;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return LGPU_OK;
}

}  // namespace

extern "C" int lgpu_tonemap_noalloc(const float* d_linrgb, uint64_t w, uint64_t h, float y_mid,
                                    float* d_out_tonemapped, uint8_t* d_out_rgb24, void* stream) {
  if (!d_linrgb || (!d_out_tonemapped && !d_out_rgb24)) return LGPU_ERR_INVALID_ARGUMENT;
  if (w == 0 || h == 0) return LGPU_OK;
  if (w > LGPU_NOALLOC_MAX_PIXELS || h > LGPU_NOALLOC_MAX_PIXELS / w) return LGPU_ERR_TOO_LARGE;
  uint64_t const n = w * h;
  if (lgpu::tonemap_partials_needed(n) > kPartials) return LGPU_ERR_TOO_LARGE;
  double* scratch = nullptr;
  int const rc = scratch_address(&scratch);
  if (rc != LGPU_OK) return rc;
  cudaStream_t const st = static_cast<cudaStream_t>(stream);
  float* exposure = reinterpret_cast<float*>(scratch + kPartials);
  cudaError_t e = lgpu::launch_tonemap(d_linrgb, n, y_mid, scratch, kPartials, exposure, d_out_tonemapped,
                                       d_out_rgb24, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? LGPU_OK : LGPU_ERR_CUDA;
}
