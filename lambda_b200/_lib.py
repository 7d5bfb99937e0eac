"""ctypes binding of liblambda_gpu.so (include/lambda_gpu.h).

The structures below mirror the C declarations field for field.  Loading the
library never falls back to anything: if the shared object is missing or
does not export the ABI, an ImportError-style RuntimeError is raised.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblambda_gpu.so")

c_float_p = ctypes.POINTER(ctypes.c_float)
c_uint32_p = ctypes.POINTER(ctypes.c_uint32)
c_uint8_p = ctypes.POINTER(ctypes.c_uint8)

# lgpu_status
OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_CUDA = -2
ERR_OUT_OF_MEMORY = -3
ERR_NO_SCENE = -4
ERR_UNSUPPORTED = -5
ERR_DEVICE_CHECK = -6
ERR_TIMEOUT = -7
ERR_NO_DEVICE = -8
ERR_TOO_LARGE = -9

OBJ_SPHERE, OBJ_PLANE, OBJ_TRIMESH = 0, 1, 2
MAT_LAMBERTIAN, MAT_BLINN, MAT_THINFILM, MAT_MICROFACET, MAT_EMITTER, MAT_DIREMITTER = range(6)
LIGHT_AMBIENT, LIGHT_POINT, LIGHT_DIR, LIGHT_SPHERE, LIGHT_QUADDIR = range(5)

FLAG_REFERENCE_ORDER = 0x1
FLAG_MEGAKERNEL = 0x2


class Transform(ctypes.Structure):
    _fields_ = [("M", ctypes.c_float * 16), ("M_inv", ctypes.c_float * 16)]


class Camera(ctypes.Structure):
    _fields_ = [("base_x", ctypes.c_float * 3), ("base_y", ctypes.c_float * 3),
                ("base_z", ctypes.c_float * 3), ("pos", ctypes.c_float * 3),
                ("fov", ctypes.c_float), ("dof", ctypes.c_float), ("D", ctypes.c_float),
                ("delta", ctypes.c_float), ("h", ctypes.c_float), ("w", ctypes.c_float),
                ("width", ctypes.c_uint64), ("height", ctypes.c_uint64)]


class Spectral(ctypes.Structure):
    _fields_ = [("n_bins", ctypes.c_uint32), ("hero_k", ctypes.c_uint32),
                ("lambda_inf", ctypes.c_float), ("lambda_sup", ctypes.c_float),
                ("cmf_x", c_float_p), ("cmf_y", c_float_p), ("cmf_z", c_float_p)]


class Material(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("spectrum", ctypes.c_int32 * 5),
                ("alpha", ctypes.c_float), ("p_d", ctypes.c_float), ("p_spec", ctypes.c_float),
                ("w_r", ctypes.c_float), ("w_t", ctypes.c_float), ("d", ctypes.c_float),
                ("specular", ctypes.c_float)]


class Object(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("mat", ctypes.c_uint32), ("mesh", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("T", Transform)]


class Light(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("spectrum", ctypes.c_int32), ("obj", ctypes.c_uint32),
                ("size", ctypes.c_float), ("inv_area", ctypes.c_float), ("spec", ctypes.c_float),
                ("pos", ctypes.c_float * 3), ("dir", ctypes.c_float * 3), ("T", Transform)]


class Mesh(ctypes.Structure):
    _fields_ = [("n_positions", ctypes.c_uint32), ("n_normals", ctypes.c_uint32),
                ("n_faces", ctypes.c_uint32), ("f_stride", ctypes.c_uint32),
                ("V", c_float_p), ("N", c_float_p), ("F", c_uint32_p), ("GN", c_float_p),
                ("bounds", ctypes.c_float * 6),
                ("n_nodes", ctypes.c_uint32), ("n_bbs", ctypes.c_uint32),
                ("n_prim_idxs", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("nodes", c_uint32_p), ("bbs", c_float_p), ("prim_idxs", c_uint32_p),
                ("n_trav_nodes", ctypes.c_uint32), ("n_trav_bbs", ctypes.c_uint32),
                ("n_trav_prim_idxs", ctypes.c_uint32), ("reserved2", ctypes.c_uint32),
                ("trav_nodes", c_uint32_p), ("trav_bbs", c_float_p), ("trav_prim_idxs", c_uint32_p)]


class Scene(ctypes.Structure):
    _fields_ = [("cam", Camera), ("spec", Spectral),
                ("n_objects", ctypes.c_uint32), ("n_materials", ctypes.c_uint32),
                ("n_lights", ctypes.c_uint32), ("n_meshes", ctypes.c_uint32),
                ("n_spectra", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("objects", ctypes.POINTER(Object)), ("materials", ctypes.POINTER(Material)),
                ("lights", ctypes.POINTER(Light)), ("meshes", ctypes.POINTER(Mesh)),
                ("spectra", c_float_p)]


class RenderParams(ctypes.Structure):
    _fields_ = [("spp", ctypes.c_uint32), ("max_scatterings", ctypes.c_uint32),
                ("sample_p", ctypes.c_float), ("flags", ctypes.c_uint32),
                ("seed", ctypes.c_uint64), ("spp_offset", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class Job(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("params", RenderParams), ("out", ctypes.c_void_p),
                ("x0", ctypes.c_uint32), ("y0", ctypes.c_uint32), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32)]


class WaveConfig(ctypes.Structure):
    _fields_ = [("queue_cap", ctypes.c_uint32), ("shade_block", ctypes.c_uint32),
                ("trace_per_sm", ctypes.c_uint32), ("graphs", ctypes.c_uint32),
                ("mega_items", ctypes.c_uint64)]


class Hit(ctypes.Structure):
    _fields_ = [("t", ctypes.c_float), ("obj", ctypes.c_uint32), ("face", ctypes.c_uint32),
                ("mat", ctypes.c_uint32), ("p", ctypes.c_float * 3), ("n", ctypes.c_float * 3),
                ("gn", ctypes.c_float * 3), ("front", ctypes.c_uint32)]


# lgpu_probe_shading (include/lambda_gpu.h): queries and results as numpy
# records with the C structs' layout (4-byte fields, no padding)
PROBE_BXDF, PROBE_PROB_MATERIAL, PROBE_SAMPLE_MATERIAL, PROBE_SAMPLE_LIGHT, PROBE_PROB_LIGHT, \
    PROBE_SPECTRUM = range(6)
PROBE_DTYPE = np.dtype([("op", "<u4"), ("index", "<u4"), ("lambda", "<f4", 16), ("p", "<f4", 3),
                        ("F", "<f4", 9), ("i", "<f4", 3), ("o", "<f4", 3), ("n", "<f4", 3),
                        ("front", "<u4"), ("sample_p", "<f4"), ("xi", "<f4", 4)])
PROBE_RESULT_DTYPE = np.dtype([("value", "<f4", 16), ("prob", "<f4"), ("dir", "<f4", 3),
                               ("tmax", "<f4"), ("skip", "<u4"), ("ok", "<u4"), ("n_xi", "<u4")])


class Stats(ctypes.Structure):
    _fields_ = [("last_kernel_ms", ctypes.c_double), ("rays", ctypes.c_uint64),
                ("paths", ctypes.c_uint64), ("device_checks", ctypes.c_uint32),
                ("max_stack", ctypes.c_uint32), ("nonfinite_paths", ctypes.c_uint32),
                ("launches", ctypes.c_uint32), ("node_tests", ctypes.c_uint64),
                ("tri_tests", ctypes.c_uint64), ("inst_tests", ctypes.c_uint64),
                ("upload_bytes", ctypes.c_uint64), ("kernel_ms", ctypes.c_double * 3),
                ("kernel_launches", ctypes.c_uint64 * 3), ("kernel_rays", ctypes.c_uint64 * 3),
                ("kernel_node_tests", ctypes.c_uint64 * 3), ("kernel_tri_tests", ctypes.c_uint64 * 3),
                ("kernel_inst_tests", ctypes.c_uint64 * 3), ("order_rays", ctypes.c_uint64),
                ("local_stack", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]

FLAG_KERNEL_TIMING = 0x4
FLAG_FP64_FILM = 0x8
# lgpu_scene.flags
SCENE_HOST_LAYOUT = 0x1
SCENE_REFERENCE_BVH = 0x2  # keep the reference's mesh BVHs for every traversal
KERNEL_CLOSEST, KERNEL_SHADOW, KERNEL_SHADE = 0, 1, 2


# every entry point of include/lambda_gpu.h: name -> (restype, argtypes)
_vp = ctypes.c_void_p
SIGNATURES = {
    "lgpu_abi_version": (ctypes.c_int, []),
    "lgpu_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "lgpu_destroy": (None, [_vp]),
    "lgpu_last_error": (ctypes.c_char_p, [_vp]),
    "lgpu_upload_scene": (ctypes.c_int, [_vp, ctypes.POINTER(Scene)]),
    "lgpu_upload_scenes": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.POINTER(Scene)), ctypes.c_uint32]),
    "lgpu_render_batch": (ctypes.c_int, [_vp, ctypes.POINTER(Job), ctypes.c_uint32]),
    "lgpu_render_batch_device": (ctypes.c_int, [_vp, ctypes.POINTER(Job), ctypes.c_uint32, _vp]),
    "lgpu_update_materials": (ctypes.c_int, [_vp, ctypes.POINTER(Scene)]),
    "lgpu_render": (ctypes.c_int, [_vp, ctypes.POINTER(RenderParams), _vp]),
    "lgpu_render_device": (ctypes.c_int, [_vp, ctypes.POINTER(RenderParams), _vp, _vp]),
    "lgpu_adjoint": (ctypes.c_int, [_vp, ctypes.POINTER(RenderParams), _vp, _vp, _vp, _vp]),
    "lgpu_adjoint_device": (ctypes.c_int, [_vp, ctypes.POINTER(RenderParams), _vp, _vp, _vp, _vp, _vp]),
    "lgpu_get_wave_config": (ctypes.c_int, [_vp, ctypes.POINTER(WaveConfig)]),
    "lgpu_set_wave_config": (ctypes.c_int, [_vp, ctypes.POINTER(WaveConfig)]),
    "lgpu_autotune_batch": (ctypes.c_int, [_vp, ctypes.POINTER(Job), ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.POINTER(WaveConfig)]),
    "lgpu_trace_closest": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, ctypes.c_uint32, _vp]),
    "lgpu_trace_any": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_uint64, ctypes.c_uint32, _vp]),
    "lgpu_probe_shading": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, _vp]),
    "lgpu_tonemap": (ctypes.c_int, [_vp, _vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float,
                                    _vp, _vp]),
    "lgpu_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(Stats)]),
    "lgpu_tonemap_noalloc": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float,
                                            _vp, _vp, _vp]),
    "lgpu_build_bvh": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, ctypes.c_uint32, ctypes.c_uint32,
                                      _vp, c_uint32_p, _vp, c_uint32_p, _vp, c_uint32_p]),
    "lgpu_build_traversal_bvh": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, ctypes.c_uint32, ctypes.c_uint32,
                                                _vp, c_uint32_p, _vp, c_uint32_p, _vp, c_uint32_p]),
    "lgpu_build_bvh_device": (ctypes.c_int, [_vp, _vp, ctypes.c_uint32, _vp, ctypes.c_uint32, ctypes.c_uint32,
                                             _vp, c_uint32_p, _vp, c_uint32_p, _vp, c_uint32_p]),
}

# LGPU_ABI_VERSION of include/lambda_gpu.h
ABI_VERSION = 4

_lib = None


def lib():
    """The loaded library; raises if it is missing (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m lambda_b200.build` "
            "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if L.lgpu_abi_version() != ABI_VERSION:
        raise RuntimeError("liblambda_gpu.so ABI version mismatch")
    _lib = L
    return L


class LgpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"lgpu error {code}: {msg}")
        self.code = code


def check(ctx, rc, what=""):
    if rc != OK:
        msg = lib().lgpu_last_error(ctx) if ctx else b""
        raise LgpuError(rc, (what + ": " if what else "") + (msg or b"").decode(errors="replace"))
