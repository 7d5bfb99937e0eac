"""TEST INFRASTRUCTURE ONLY — ctypes access to the C restatement oracle
(oracle/lambda_oracle.c, built into oracle/_build/liboracle.so)."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")

RNG_MT19937 = 0
RNG_PCG = 1

_vp = ctypes.c_void_p
_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        L.oracle_intersect.argtypes = [_vp, _vp, ctypes.c_uint64, _vp]
        L.oracle_intersect.restype = None
        L.oracle_render_rows.argtypes = [_vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                                         ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32,
                                         ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _vp, _vp]
        L.oracle_render_rows.restype = None
        L.oracle_mt_flt.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _vp]
        L.oracle_mt_u64.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _vp]
        L.oracle_set_mt_arg_order.argtypes = [ctypes.c_int]
        L.oracle_max_threads.restype = ctypes.c_int
        L.oracle_unit_spectrum.argtypes = [_vp, ctypes.c_uint32, _vp, _vp]
        L.oracle_unit_spectrum.restype = None
        L.oracle_unit_add_hero.argtypes = [_vp, _vp, _vp, _vp]
        L.oracle_unit_add_hero.restype = None
        L.oracle_unit_bxdf.argtypes = [_vp, ctypes.c_uint32, _vp, _vp, _vp, _vp, ctypes.c_int, _vp]
        L.oracle_unit_bxdf.restype = None
        L.oracle_unit_prob_for_material.argtypes = [_vp, ctypes.c_float, _vp, _vp, _vp, ctypes.c_float]
        L.oracle_unit_prob_for_material.restype = ctypes.c_float
        L.oracle_unit_sample_material.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_uint64, ctypes.c_float,
                                                  _vp, _vp, _vp]
        L.oracle_unit_sample_material.restype = ctypes.c_int
        L.oracle_unit_sample_light.argtypes = [_vp, ctypes.c_uint32, _vp, _vp, ctypes.c_uint64, _vp, _vp,
                                               _vp]
        L.oracle_unit_sample_light.restype = None
        L.oracle_unit_prob_for_light.argtypes = [_vp, ctypes.c_uint32, _vp]
        L.oracle_unit_prob_for_light.restype = ctypes.c_float
        _lib = L
    return _lib


class Oracle:
    """The restatement over a scene: a SceneData/FlatScene of lambda_b200, or
    a pointer to an lgpu_scene exported by the reference harness."""

    def __init__(self, scene):
        from lambda_b200.scene import FlatScene, SceneData
        self.L = lib()
        if isinstance(scene, SceneData):
            scene = FlatScene(scene)
        if isinstance(scene, FlatScene):
            self.flat = scene
            self.ptr = ctypes.addressof(scene.scene)
            cam = scene.scene.cam
        else:  # an lgpu_scene pointer (int) and its camera size
            self.flat = None
            self.ptr = scene[0]
            cam = None
            self.width, self.height = scene[1], scene[2]
        if cam is not None:
            self.width, self.height = int(cam.width), int(cam.height)

    def intersect(self, rays):
        from lambda_b200 import _lib as LG
        from lambda_b200.renderer import hits_to_numpy
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = (LG.Hit * max(rays.shape[0], 1))()
        self.L.oracle_intersect(self.ptr, rays.ctypes.data, rays.shape[0], ctypes.addressof(out))
        return hits_to_numpy(out, rays.shape[0])

    def render_rows(self, spp, max_scatter, sample_p, row0, row1, rng=RNG_MT19937, seed=0,
                    spp_offset=0, fp64=False):
        n = (row1 - row0) * self.width * 3
        if fp64:
            out = np.zeros(n, np.float64)
            self.L.oracle_render_rows(self.ptr, spp, max_scatter, sample_p, rng, seed, spp_offset,
                                      row0, row1, 1, None, out.ctypes.data)
        else:
            out = np.zeros(n, np.float32)
            self.L.oracle_render_rows(self.ptr, spp, max_scatter, sample_p, rng, seed, spp_offset,
                                      row0, row1, 0, out.ctypes.data, None)
        return out.reshape(row1 - row0, self.width, 3)

    def render(self, spp, max_scatter, sample_p, rng=RNG_MT19937, seed=0, fp64=False):
        """The full image in Renderer::render's layout (row 0 at the top)."""
        band = self.render_rows(spp, max_scatter, sample_p, 0, self.height, rng, seed, 0, fp64)
        return band[::-1].copy()


def mt_flt(seed, n):
    out = np.zeros(n, np.float32)
    lib().oracle_mt_flt(seed, n, out.ctypes.data)
    return out


def mt_u64(seed, n):
    out = np.zeros(n, np.uint64)
    lib().oracle_mt_u64(seed, n, out.ctypes.data)
    return out
