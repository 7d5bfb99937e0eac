"""TEST INFRASTRUCTURE ONLY — ctypes access to the reference renderer.

Loads oracle/_ref/libref.so (the reference's own sources compiled by
oracle/Makefile with ref_harness.cpp).  Only tests, the smoke check and the
CPU-baseline leg of bench.py use this module, always as the checker.

The reference reads its colour tables at start-up from ../lib/numli/data
relative to the working directory (cg.hpp:329-337); where that directory
does not exist the tables are zero, so load() first installs the tables
(bit-identical to the reference's, see tests/test_scene_loader.py).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_EXACT = os.path.join(HERE, "_ref", "libref.so")
LIB_FAST = os.path.join(HERE, "_ref", "libref_fast.so")
# the same sources built at the configurations' spectral setting (4 hero
# wavelengths, 81 bins on 380-780 nm; oracle/Makefile)
LIB_K4_EXACT = os.path.join(HERE, "_ref", "libref_k4.so")
LIB_K4_FAST = os.path.join(HERE, "_ref", "libref_k4_fast.so")


def _path(fast, k4):
    if k4:
        return LIB_K4_FAST if fast else LIB_K4_EXACT
    return LIB_FAST if fast else LIB_EXACT

_vp = ctypes.c_void_p


class RefHit(ctypes.Structure):
    """ref_hitinfo of ref_harness.cpp (hitinfo, cg.hpp:1138-1149)."""
    _fields_ = [("z", ctypes.c_float), ("p", ctypes.c_float * 3), ("Fx", ctypes.c_float * 3),
                ("Fy", ctypes.c_float * 3), ("Fz", ctypes.c_float * 3), ("gn", ctypes.c_float * 3),
                ("front", ctypes.c_uint32), ("mat", ctypes.c_uint32), ("obj", ctypes.c_uint32)]


_SIGS = {
    "ref_n_bins": (ctypes.c_int, []),
    "ref_lambda_range": (None, [_vp]),
    "ref_hero_samples": (ctypes.c_int, []),
    "ref_get_tables": (None, [_vp]),
    "ref_set_tables": (None, [_vp]),
    "ref_coef_from_samples": (None, [_vp, _vp, ctypes.c_uint64, _vp]),
    "ref_load": (_vp, [ctypes.c_char_p]),
    "ref_free": (None, [_vp]),
    "ref_export": (_vp, [_vp]),
    "ref_camera": (None, [_vp, _vp]),
    "ref_intersect": (None, [_vp, _vp, ctypes.c_uint64, _vp]),
    "ref_occluded": (None, [_vp, _vp, _vp, _vp, ctypes.c_uint64, _vp]),
    "ref_render": (None, [_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float, _vp]),
    "ref_render_rows": (None, [_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float,
                               ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _vp, _vp]),
    "ref_render_rows_seeded": (None, [_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float,
                                      ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64,
                                      _vp, _vp]),
    "ref_trace_path": (None, [_vp, _vp, _vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float,
                              _vp]),
    "ref_rng_flt": (None, [ctypes.c_uint64, ctypes.c_uint64, _vp]),
    "ref_rng_u64": (None, [ctypes.c_uint64, ctypes.c_uint64, _vp]),
    "ref_rng_mixed": (None, [ctypes.c_uint64, ctypes.c_uint64, _vp, _vp, _vp]),
    "ref_camera_ray": (None, [_vp, ctypes.c_float, ctypes.c_float, ctypes.c_uint64, _vp]),
    "ref_hero": (ctypes.c_float, [ctypes.c_uint64, _vp]),
    "ref_eval_spectrum": (None, [_vp, _vp, _vp]),
    "ref_add_hero": (None, [_vp, _vp, _vp]),
    "ref_coef_to_linrgb": (None, [_vp, _vp]),
    "ref_bxdf": (None, [_vp, ctypes.c_uint32, _vp, _vp, _vp, _vp, ctypes.c_int, _vp]),
    "ref_sample_material": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(RefHit), _vp, ctypes.c_uint64,
                                           ctypes.c_float, _vp, _vp, _vp]),
    "ref_prob_for_material": (ctypes.c_float, [_vp, ctypes.c_float, ctypes.POINTER(RefHit), _vp,
                                               _vp, ctypes.c_float]),
    "ref_sample_light": (None, [_vp, ctypes.c_uint32, _vp, ctypes.POINTER(RefHit), ctypes.c_uint64,
                                _vp, _vp, _vp]),
    "ref_prob_for_light": (ctypes.c_float, [_vp, ctypes.c_uint32, _vp]),
    "ref_tonemap": (None, [_vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_float, _vp, _vp]),
    "ref_max_threads": (ctypes.c_int, []),
}

_libs = {}


def available(fast=False, k4=False):
    return os.path.exists(_path(fast, k4))


def lib(fast=False, k4=False):
    path = _path(fast, k4)
    if path in _libs:
        return _libs[path]
    L = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _install_tables(L)
    _libs[path] = L
    return L


def spectral_config(L):
    """The library's compiled-in spectral discretisation as a
    lambda_b200.scene.SpectralConfig."""
    from lambda_b200.scene import SpectralConfig
    r = np.zeros(2, np.float32)
    L.ref_lambda_range(r.ctypes.data)
    return SpectralConfig(n_bins=L.ref_n_bins(), lambda_inf=float(r[0]), lambda_sup=float(r[1]),
                          hero_k=L.ref_hero_samples())


def _install_tables(L):
    """Installs the CMF/BT.709 tables if start-up found no data files."""
    from lambda_b200.scene import cie_tables
    cur = np.zeros(6 * L.ref_n_bins(), np.float32)
    L.ref_get_tables(cur.ctypes.data)
    if not np.any(cur):
        t = np.concatenate(cie_tables(spectral_config(L))).astype(np.float32)
        L.ref_set_tables(t.ctypes.data)


class RefScene:
    """A scene loaded by the reference loader."""

    def __init__(self, nls_path, fast=False, k4=False):
        self.L = lib(fast, k4)
        self.h = self.L.ref_load(os.path.abspath(nls_path).encode())
        if not self.h:
            raise RuntimeError(f"reference loader failed on {nls_path}")
        wh = np.zeros(2, np.uint64)
        self.L.ref_camera(self.h, wh.ctypes.data)
        self.width, self.height = int(wh[0]), int(wh[1])

    def close(self):
        if self.h:
            self.L.ref_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def intersect(self, rays):
        from lambda_b200.renderer import hits_to_numpy
        from lambda_b200 import _lib as LG
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = (LG.Hit * max(rays.shape[0], 1))()
        self.L.ref_intersect(self.h, rays.ctypes.data, rays.shape[0], ctypes.addressof(out))
        return hits_to_numpy(out, rays.shape[0])

    def occluded(self, rays, tmax, skip):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        tmax = np.ascontiguousarray(tmax, np.float32)
        skip = np.ascontiguousarray(skip, np.uint32)
        out = np.zeros(rays.shape[0], np.uint8)
        self.L.ref_occluded(self.h, rays.ctypes.data, tmax.ctypes.data, skip.ctypes.data,
                            rays.shape[0], out.ctypes.data)
        return out.astype(bool)

    def render(self, spp, max_scatter, sample_p):
        out = np.zeros((self.height, self.width, 3), np.float32)
        self.L.ref_render(self.h, spp, max_scatter, sample_p, out.ctypes.data)
        return out

    def render_rows(self, spp, max_scatter, sample_p, row0, row1, fp64=False, seed_base=0):
        """Scene rows [row0, row1) in scene order (not flipped).  Pixel
        (i, j) draws from the reference's RNG seeded seed_base + i*w + j
        (seed_base 0: Renderer::render's own streams)."""
        n = (row1 - row0) * self.width * 3
        if fp64:
            out = np.zeros(n, np.float64)
            self.L.ref_render_rows_seeded(self.h, spp, max_scatter, sample_p, row0, row1, 1, seed_base,
                                          None, out.ctypes.data)
        else:
            out = np.zeros(n, np.float32)
            self.L.ref_render_rows_seeded(self.h, spp, max_scatter, sample_p, row0, row1, 0, seed_base,
                                          out.ctypes.data, None)
        return out.reshape(row1 - row0, self.width, 3)

    def render_fp64(self, spp, max_scatter, sample_p):
        """Full image with FP64 film accumulation, in Renderer::render's
        layout (row 0 at the top)."""
        band = self.render_rows(spp, max_scatter, sample_p, 0, self.height, fp64=True)
        return band[::-1].copy()
