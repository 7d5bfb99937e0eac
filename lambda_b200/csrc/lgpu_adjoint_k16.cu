// lgpu_adjoint_k16.cu — path-replay adjoint kernels for 16 hero wavelengths per path.
#include "lgpu_adjoint.cuh"

namespace lgpu {
template cudaError_t launch_adjoint_k<16>(const DevScene&, const RenderArgs&, WaveState*, uint64_t, float*,
                                         const AdjointArgs&, DevCounters*, cudaStream_t, WaveLaunch*);
}  // namespace lgpu
