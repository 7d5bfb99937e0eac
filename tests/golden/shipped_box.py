"""Golden fixture of the reference's shipped scene bin/scenes/box.nls
(spheres, planes, RGB and measured spectra, a sphere light).

    python -m tests.golden.shipped_box        # regenerate shipped_box.npz

Generation needs the reference tree (oracle/refpath.py) and the reference
build oracle/_ref/libref.so; it runs only here, never in the tests.  It
loads the scene with the reference's own loader (cg.hpp:2455-2470) from the
reference's bin/ directory, flattens it through the drop-in flattener, and
stores:
  * the flattened scene (camera, spectral table, objects, materials,
    lights, spectra: the lgpu_scene arrays the device takes);
  * N_ROWS image rows of the reference's own Renderer::render streams at
    REF_SPP samples per pixel (float film, as the reference renders);
  * the same rows as an FP64-accumulated ORACLE_SPP-sample oracle drawn
    from streams disjoint from the reference's render (seed base w*h);
  * the error statistics of MSE_RENDERS independent reference renders of
    those rows at REF_SPP (seed bases 2*w*h, 3*w*h, ...) against the stored
    oracle, per channel: the median and 90th percentile of |img - oracle| /
    RMS(oracle) pooled over the renders' pixels, and the median of their
    relative MSEs.
The GPU test (tests/test_gpu_render.py) rebuilds the scene from the arrays,
renders it on the device and compares against these rows.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "shipped_box.npz")
REF_SPP = 64
ORACLE_SPP = 1024
BOUNCES = 8
SAMPLE_P = 0.8
N_ROWS = 12
MSE_RENDERS = 16


def _raw(ptr, n, ctype):
    return np.frombuffer(ctypes.string_at(ptr, n * ctypes.sizeof(ctype)), np.uint8).copy()


def generate():
    from lambda_b200 import _lib as L
    from oracle import refharness, refpath
    bindir = refpath.path("bin")
    cwd = os.getcwd()
    os.chdir(bindir)  # the reference resolves the scene's files and its tables from here
    try:
        ref = refharness.RefScene(os.path.join("scenes", "box.nls"))
    finally:
        os.chdir(cwd)
    sc = ctypes.cast(ref.L.ref_export(ref.h), ctypes.POINTER(L.Scene)).contents
    assert sc.n_meshes == 0
    nb = int(sc.spec.n_bins)
    cmf = np.stack([np.ctypeslib.as_array(p, (nb,)).copy() for p in (sc.spec.cmf_x, sc.spec.cmf_y,
                                                                         sc.spec.cmf_z)])
    W, H = int(sc.cam.width), int(sc.cam.height)
    rows = np.linspace(0, H - 1, N_ROWS).round().astype(np.int64)
    img_ref = np.stack([ref.render_rows(REF_SPP, BOUNCES, SAMPLE_P, r, r + 1)[0] for r in rows])
    img_orc = np.stack([ref.render_rows(ORACLE_SPP, BOUNCES, SAMPLE_P, r, r + 1, fp64=True,
                                        seed_base=W * H)[0] for r in rows])
    orc = img_orc.astype(np.float32).astype(np.float64)
    scale = np.sqrt(np.mean(orc ** 2, axis=(0, 1)))
    mses, errs = [], []
    for k in range(MSE_RENDERS):
        img = np.stack([ref.render_rows(REF_SPP, BOUNCES, SAMPLE_P, r, r + 1, seed_base=(2 + k) * W * H)[0]
                        for r in rows]).astype(np.float64)
        mses.append(np.sum((img - orc) ** 2, axis=(0, 1)) / np.sum(orc ** 2, axis=(0, 1)))
        errs.append((np.abs(img - orc) / scale).reshape(-1, 3))
    np.savez_compressed(
        PATH, camera=_raw(ctypes.addressof(sc.cam), 1, L.Camera),
        spec=np.array([nb, sc.spec.hero_k], np.uint32),
        lam=np.array([sc.spec.lambda_inf, sc.spec.lambda_sup], np.float32), cmf=cmf.astype(np.float32),
        objects=_raw(ctypes.addressof(sc.objects.contents), sc.n_objects, L.Object),
        materials=_raw(ctypes.addressof(sc.materials.contents), sc.n_materials, L.Material),
        lights=_raw(ctypes.addressof(sc.lights.contents), sc.n_lights, L.Light),
        spectra=np.ctypeslib.as_array(sc.spectra, (sc.n_spectra * nb,)).astype(np.float32),
        rows=rows, ref=img_ref.astype(np.float32), oracle=img_orc.astype(np.float32),
        settings=np.array([REF_SPP, ORACLE_SPP, BOUNCES], np.int64),
        ref_mse_median=np.median(mses, axis=0), ref_renders=np.array([MSE_RENDERS], np.int64),
        ref_err_quantiles=np.percentile(np.concatenate(errs), [50, 90], axis=0),
        sample_p=np.array([SAMPLE_P], np.float32))
    return PATH


class FixtureScene:
    """The stored lgpu_scene; keeps every array it points to alive."""

    def __init__(self, d):
        from lambda_b200 import _lib as L

        def arr(ctype, raw):
            n = len(raw) // ctypes.sizeof(ctype)
            return (ctype * max(n, 1)).from_buffer_copy(raw.tobytes() or bytes(ctypes.sizeof(ctype))), n

        self.cmf = np.ascontiguousarray(d["cmf"], np.float32)
        self.spectra = np.ascontiguousarray(d["spectra"], np.float32)
        self.objects, no = arr(L.Object, d["objects"])
        self.materials, nm = arr(L.Material, d["materials"])
        self.lights, nl = arr(L.Light, d["lights"])
        self.meshes = (L.Mesh * 1)()
        s = L.Scene()
        s.cam = L.Camera.from_buffer_copy(d["camera"].tobytes())
        s.spec.n_bins, s.spec.hero_k = (int(x) for x in d["spec"])
        s.spec.lambda_inf, s.spec.lambda_sup = (float(x) for x in d["lam"])
        s.spec.cmf_x, s.spec.cmf_y, s.spec.cmf_z = (self.cmf[k].ctypes.data_as(L.c_float_p) for k in range(3))
        s.n_objects, s.n_materials, s.n_lights, s.n_meshes = no, nm, nl, 0
        s.n_spectra = self.spectra.size // int(d["spec"][0])
        s.objects, s.materials, s.lights, s.meshes = self.objects, self.materials, self.lights, self.meshes
        s.spectra = self.spectra.ctypes.data_as(L.c_float_p)
        self.scene = s

    def ptr(self):
        return ctypes.pointer(self.scene)


def load():
    """(FixtureScene, the npz contents)."""
    d = dict(np.load(PATH))
    return FixtureScene(d), d


if __name__ == "__main__":
    print(generate())
