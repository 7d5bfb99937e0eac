// lgpu_batch_k8.cu — batched render kernels for 8 hero wavelengths per path.
#include "lgpu_render.cuh"

namespace lgpu {
template cudaError_t launch_batch_k<8>(const DevJob*, const uint64_t*, const uint32_t*, uint32_t, uint64_t,
                                       uint64_t, bool, WaveState*, DevCounters*, cudaStream_t, WaveLaunch*);
}  // namespace lgpu
