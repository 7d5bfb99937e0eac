"""The Python host's .nls loader (lambda_b200.scene) against the reference's
loader (load::loadNLS, cg.hpp:2455) flattened by the C++ drop-in flattener:
every flattened array must be bit-identical — camera, spectra (CSV box
averages, RGB through the BT.709 basis), CMF tables, materials incl.
blinn::init, transforms, lights, meshes with their BVH."""
import ctypes
import os

import numpy as np
import pytest

from lambda_b200 import _lib as L
from lambda_b200.scene import flatten, load_nls
from oracle import refharness, refpath

pytestmark = pytest.mark.skipif(not refharness.available(), reason="reference harness not built")


def _arr(ptr, n, dt):
    if n == 0:
        return np.zeros(0, dt)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt).copy()


def _f32(x):
    return np.atleast_1d(np.asarray(x, np.float32)).view(np.uint32)


def compare_scenes(rs, ms):
    bad = []

    def chk(name, a, b):
        a, b = np.atleast_1d(np.asarray(a)), np.atleast_1d(np.asarray(b))
        if a.shape != b.shape or not np.array_equal(a, b):
            bad.append(name)

    for f in ("base_x", "base_y", "base_z", "pos"):
        chk("cam." + f, _f32(getattr(rs.cam, f)[:]), _f32(getattr(ms.cam, f)[:]))
    for f in ("fov", "dof", "D", "delta", "h", "w"):
        chk("cam." + f, _f32(getattr(rs.cam, f)), _f32(getattr(ms.cam, f)))
    chk("cam.wh", [rs.cam.width, rs.cam.height], [ms.cam.width, ms.cam.height])
    chk("counts", [rs.n_objects, rs.n_materials, rs.n_lights, rs.n_meshes, rs.n_spectra],
        [ms.n_objects, ms.n_materials, ms.n_lights, ms.n_meshes, ms.n_spectra])
    if bad:
        return bad
    nb = rs.spec.n_bins
    chk("spectra", _f32(_arr(rs.spectra, rs.n_spectra * nb, np.float32)),
        _f32(_arr(ms.spectra, ms.n_spectra * nb, np.float32)))
    for c in ("cmf_x", "cmf_y", "cmf_z"):
        chk(c, _f32(_arr(getattr(rs.spec, c), nb, np.float32)),
            _f32(_arr(getattr(ms.spec, c), nb, np.float32)))
    for i in range(rs.n_materials):
        a, b = rs.materials[i], ms.materials[i]
        chk(f"mat{i}", [a.type] + list(a.spectrum), [b.type] + list(b.spectrum))
        chk(f"mat{i}.f", _f32([a.alpha, a.p_d, a.p_spec, a.w_r, a.w_t, a.d, a.specular]),
            _f32([b.alpha, b.p_d, b.p_spec, b.w_r, b.w_t, b.d, b.specular]))
    for i in range(rs.n_objects):
        a, b = rs.objects[i], ms.objects[i]
        chk(f"obj{i}", [a.type, a.mat, a.mesh], [b.type, b.mat, b.mesh])
        chk(f"obj{i}.T", _f32(a.T.M[:] + a.T.M_inv[:]), _f32(b.T.M[:] + b.T.M_inv[:]))
    for i in range(rs.n_lights):
        a, b = rs.lights[i], ms.lights[i]
        chk(f"light{i}", [a.type, a.spectrum, a.obj], [b.type, b.spectrum, b.obj])
        chk(f"light{i}.f", _f32([a.size, a.inv_area, a.spec] + a.pos[:] + a.dir[:] + a.T.M[:] + a.T.M_inv[:]),
            _f32([b.size, b.inv_area, b.spec] + b.pos[:] + b.dir[:] + b.T.M[:] + b.T.M_inv[:]))
    for i in range(rs.n_meshes):
        a, b = rs.meshes[i], ms.meshes[i]
        chk(f"mesh{i}.n", [a.n_positions, a.n_normals, a.n_faces, a.n_nodes, a.n_bbs, a.n_prim_idxs],
            [b.n_positions, b.n_normals, b.n_faces, b.n_nodes, b.n_bbs, b.n_prim_idxs])
        chk(f"mesh{i}.V", _f32(_arr(a.V, 3 * a.n_positions, np.float32)),
            _f32(_arr(b.V, 3 * b.n_positions, np.float32)))
        chk(f"mesh{i}.N", _f32(_arr(a.N, 3 * a.n_normals, np.float32)),
            _f32(_arr(b.N, 3 * b.n_normals, np.float32)))
        Fa = _arr(a.F, a.f_stride * a.n_faces, np.uint32).reshape(-1, a.f_stride)[:, :6]
        Fb = _arr(b.F, b.f_stride * b.n_faces, np.uint32).reshape(-1, b.f_stride)[:, :6]
        chk(f"mesh{i}.F", Fa, Fb)
        chk(f"mesh{i}.GN", _f32(_arr(a.GN, 3 * a.n_faces, np.float32)),
            _f32(_arr(b.GN, 3 * b.n_faces, np.float32)))
        chk(f"mesh{i}.bounds", _f32(a.bounds[:]), _f32(b.bounds[:]))
        na = _arr(a.nodes, 2 * a.n_nodes, np.uint32)
        chk(f"mesh{i}.nodes", na, _arr(b.nodes, 2 * b.n_nodes, np.uint32))
        chk(f"mesh{i}.prims", _arr(a.prim_idxs, a.n_prim_idxs, np.uint32),
            _arr(b.prim_idxs, b.n_prim_idxs, np.uint32))
        # child-box records in use (the reference never initialises the
        # first n_interior records of bbs, cg.hpp:690)
        na = na.reshape(-1, 2)
        used = na[(na[:, 1] & 1) == 0, 0]
        ba = _arr(a.bbs, 48 * a.n_bbs, np.float32).reshape(-1, 48)[used]
        bb = _arr(b.bbs, 48 * b.n_bbs, np.float32).reshape(-1, 48)[used]
        chk(f"mesh{i}.bbs", _f32(ba), _f32(bb))
    return bad


@pytest.mark.parametrize("k4", [False, pytest.param(True, marks=pytest.mark.skipif(
    not refharness.available(k4=True), reason="K=4 reference build absent"))])
@pytest.mark.parametrize("which", ["mixed_nls", "mixed2_nls", "box_nls"])
def test_loader_matches_reference(which, k4, request):
    """Every flattened array of the loader mirror equals the reference
    loader's, at the reference's spectral constants and (k4) at the
    configurations' 4 hero wavelengths, 81 bins on 380-780 nm."""
    nls = request.getfixturevalue(which)
    ref = refharness.RefScene(nls, k4=k4)
    rs = ctypes.cast(ref.L.ref_export(ref.h), ctypes.POINTER(L.Scene)).contents
    fs = flatten(load_nls(nls, refharness.spectral_config(ref.L)))
    assert int(fs.scene.spec.n_bins) == (81 if k4 else 80)
    assert compare_scenes(rs, fs.scene) == []


@pytest.mark.skipif(not refpath.present("bin"), reason="reference assets absent")
def test_loader_matches_reference_on_shipped_box_scene():
    """bin/scenes/box.nls: spheres, planes, RGB spectra, a sphere light."""
    nls = refpath.path("bin", "scenes", "box.nls")
    cwd = os.getcwd()
    os.chdir(refpath.path("bin"))
    try:
        ref = refharness.RefScene(os.path.relpath(nls))
    finally:
        os.chdir(cwd)
    rs = ctypes.cast(ref.L.ref_export(ref.h), ctypes.POINTER(L.Scene)).contents
    fs = flatten(load_nls(nls, base_dir=refpath.path("bin")))
    assert compare_scenes(rs, fs.scene) == []


@pytest.mark.parametrize("k4", [False, True])
def test_cie_tables_match_reference(k4):
    """The CMF and BT.709 tables built from lambda_b200/data equal the
    reference's start-up tables (read from lib/numli/data when present): 80
    bins on 400-720 nm, and (k4) 81 bins on 380-780 nm."""
    from lambda_b200.scene import cie_tables
    if not refpath.present("lib/numli/data"):
        pytest.skip("reference data files absent")
    if not refharness.available(k4=k4):
        pytest.skip("reference build absent")
    import subprocess
    import sys
    path = refharness.LIB_K4_EXACT if k4 else refharness.LIB_EXACT
    n = 6 * (81 if k4 else 80)
    code = ("import ctypes,numpy as np;L=ctypes.CDLL(%r);o=np.zeros(%d,np.float32);"
            "L.ref_get_tables(ctypes.c_void_p(o.ctypes.data));print(o.tobytes().hex())" % (path, n))
    out = subprocess.run([sys.executable, "-c", code], cwd=refpath.path("bin"), check=True,
                         capture_output=True, text=True).stdout.strip()
    ref = np.frombuffer(bytes.fromhex(out), np.float32)
    assert np.any(ref != 0)
    cfg = refharness.spectral_config(refharness.lib(k4=k4))
    mine = np.concatenate(cie_tables(cfg)).astype(np.float32)
    assert np.array_equal(ref.view(np.uint32), mine.view(np.uint32))
