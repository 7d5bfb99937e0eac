// lgpu_render_k4.cu — render kernels for 4 hero wavelengths per path.
#include "lgpu_render.cuh"

namespace lgpu {
template cudaError_t launch_render_k<4>(const DevScene&, const RenderArgs&, WaveState*, float*,
                                        DevCounters*, cudaStream_t, WaveLaunch*);
}  // namespace lgpu
