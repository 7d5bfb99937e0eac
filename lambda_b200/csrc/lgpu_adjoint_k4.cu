// lgpu_adjoint_k4.cu — path-replay adjoint kernels for 4 hero wavelengths per path.
#include "lgpu_adjoint.cuh"

namespace lgpu {
template cudaError_t launch_adjoint_k<4>(const DevScene&, const RenderArgs&, WaveState*, uint64_t, float*,
                                         const AdjointArgs&, DevCounters*, cudaStream_t, WaveLaunch*);
}  // namespace lgpu
