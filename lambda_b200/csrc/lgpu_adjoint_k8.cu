// lgpu_adjoint_k8.cu — path-replay adjoint kernels for 8 hero wavelengths per path.
#include "lgpu_adjoint.cuh"

namespace lgpu {
template cudaError_t launch_adjoint_k<8>(const DevScene&, const RenderArgs&, WaveState*, uint64_t, float*,
                                         const AdjointArgs&, DevCounters*, cudaStream_t, WaveLaunch*);
}  // namespace lgpu
