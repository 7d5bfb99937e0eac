"""lambda_b200 — B200 (sm_100a) spectral path tracing for lambda's render call.

The compute path is liblambda_gpu.so (CUDA, C ABI in include/lambda_gpu.h);
this package is the Python host around it: the .nls scene loader mirror
(scene), the Renderer mirror (renderer) and the synthetic benchmark scenes
(synth).
"""
from .renderer import Context, Renderer, Rendering
from .scene import SpectralConfig, load_nls, flatten, REFERENCE_SPECTRAL

__all__ = ["Context", "Renderer", "Rendering", "SpectralConfig", "load_nls", "flatten",
           "REFERENCE_SPECTRAL"]
