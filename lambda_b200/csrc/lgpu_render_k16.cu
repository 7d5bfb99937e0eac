// lgpu_render_k16.cu — render kernels for 16 hero wavelengths per path.
#include "lgpu_render.cuh"

namespace lgpu {
template cudaError_t launch_render_k<16>(const DevScene&, const RenderArgs&, WaveState*, float*,
                                        DevCounters*, cudaStream_t, WaveLaunch*);
}  // namespace lgpu
