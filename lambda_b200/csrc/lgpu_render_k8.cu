// lgpu_render_k8.cu — render kernels for 8 hero wavelengths per path.
#include "lgpu_render.cuh"

namespace lgpu {
template cudaError_t launch_render_k<8>(const DevScene&, const RenderArgs&, WaveState*, float*,
                                        DevCounters*, cudaStream_t, WaveLaunch*);
}  // namespace lgpu
