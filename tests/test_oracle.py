"""Pins the C restatement oracle (oracle/lambda_oracle.c) to the reference
itself (oracle/_ref, built from the reference's sources).

The reference ships no tests or golden vectors, so the restatement is pinned
against the reference's own code run here: its random streams, its
closest-hit results and whole rendered images must be bit-identical.
"""
import numpy as np
import pytest

from lambda_b200.scene import flatten, load_nls
from oracle import refharness
from oracle import restatement as R
from tests import raysets

pytestmark = pytest.mark.skipif(not refharness.available(), reason="reference harness not built")

# the reference built at its own spectral constants (16 hero wavelengths, 80
# bins on 400-720 nm) and at the configurations' (4, 81 on 380-780 nm)
BUILDS = [False, pytest.param(True, marks=pytest.mark.skipif(not refharness.available(k4=True),
                                                             reason="K=4 reference build absent"))]


def _load(nls, k4):
    """The scene through the loader mirror with the build's spectral
    setting, and through the reference build's own loader."""
    ref = refharness.RefScene(nls, k4=k4)
    return load_nls(nls, refharness.spectral_config(ref.L)), ref


def test_mt19937_streams_match_reference():
    L = refharness.lib()
    for seed in (0, 1, 42, 1279 * 1280 + 7):
        a = np.zeros(2000, np.float32)
        L.ref_rng_flt(seed, 2000, a.ctypes.data)
        assert np.array_equal(a, R.mt_flt(seed, 2000))
        b = np.zeros(700, np.uint64)
        L.ref_rng_u64(seed, 700, b.ctypes.data)
        assert np.array_equal(b, R.mt_u64(seed, 700))


@pytest.mark.parametrize("which", ["mixed_nls", "mixed2_nls", "box_nls"])
def test_intersect_bit_exact(which, request):
    nls = request.getfixturevalue(which)
    sc = load_nls(nls)
    ref = refharness.RefScene(nls)
    o = R.Oracle(flatten(sc))
    rays = raysets.camera_rays(sc, 64, seed=3)
    h = ref.intersect(rays)
    rays = np.concatenate([rays, raysets.bounce_rays(h, 4),
                           raysets.random_rays([-4, -4, 0.01], [4, 4, 4], 5000, 6)])
    h = ref.intersect(rays)
    g = o.intersect(rays)
    for f in ("t", "obj", "mat", "p", "n", "gn", "front"):
        assert np.array_equal(np.ascontiguousarray(h[f]).view(np.uint32),
                              np.ascontiguousarray(g[f]).view(np.uint32)), f
    tri = (g["obj"] != 0xFFFFFFFF) & (g["face"] != 0xFFFFFFFF)
    assert tri.sum() > 0


@pytest.mark.parametrize("k4", BUILDS)
@pytest.mark.parametrize("which", ["mixed_nls", "mixed2_nls", "box_nls"])
def test_render_bit_exact_with_reference_stream(which, k4, request):
    nls = request.getfixturevalue(which)
    sc, ref = _load(nls, k4)
    assert int(sc.cfg.hero_k) == (4 if k4 else 16)
    o = R.Oracle(flatten(sc))
    R.lib().oracle_set_mt_arg_order(1)
    rows = (sc.cam.height // 3, sc.cam.height // 3 + 12)
    a = o.render_rows(4, 8, 0.8, *rows)
    b = ref.render_rows(4, 8, 0.8, *rows)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_fp64_film_close_to_float_film(mixed_nls):
    ref = refharness.RefScene(mixed_nls)
    a = ref.render_rows(8, 6, 0.8, 10, 14)
    b = ref.render_rows(8, 6, 0.8, 10, 14, fp64=True)
    assert np.allclose(a, b, rtol=1e-4, atol=1e-3)


# ---- the restatement's single functions against the reference's ------------------

def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _unit_vectors(rng, n):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


@pytest.fixture(scope="module", params=BUILDS, ids=["k16", "k4"])
def unit_scene(scene_dir, request):
    import os
    from lambda_b200 import synth
    nls = synth.mixed(os.path.join(str(scene_dir), "oracle_units"),
                      lights=("sphere", "quaddir", "point", "direction", "ambient"), width=16, seed=5)
    sc, ref = _load(nls, request.param)
    return flatten(sc), ref


def _queries(ref, rng, n):
    """Hero wavelengths, shading frames, hit points and directions, mostly
    on the side of the surface the hit faces."""
    lam = np.zeros((n, 16), np.float32)
    for t in range(n):
        ref.L.ref_hero(int(rng.integers(1, 2 ** 62)), lam[t].ctypes.data)
    z = _unit_vectors(rng, n)
    a = np.where(np.abs(z[:, :1]) < 0.9, [[1.0, 0.0, 0.0]], [[0.0, 1.0, 0.0]])
    x = np.cross(z, a)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    F = np.concatenate([x, np.cross(z, x), z], axis=1).astype(np.float32)
    front = rng.random(n) < 0.8
    nz = z * np.where(front, 1.0, -1.0)[:, None]

    def toward():
        d = _unit_vectors(rng, n)
        flip = (rng.random(n) < 0.75) & (np.sum(d * nz, axis=1) < 0)
        d[flip] *= -1
        return d.astype(np.float32)

    p = rng.uniform([-2, -2, 0], [2, 2, 2], (n, 3)).astype(np.float32)
    return lam, F, front, nz.astype(np.float32), p, toward(), toward()


def _hits(F, front, p, mat):
    hs = []
    for t in range(len(F)):
        h = refharness.RefHit()
        h.z = 0.0
        h.p[:] = p[t].tolist()
        h.Fx[:], h.Fy[:], h.Fz[:] = F[t, 0:3].tolist(), F[t, 3:6].tolist(), F[t, 6:9].tolist()
        h.gn[:] = F[t, 6:9].tolist()
        h.front = int(front[t])
        h.mat = mat
        h.obj = 0xFFFFFFFF
        hs.append(h)
    return hs


def test_unit_functions_bit_exact(unit_scene):
    """BxDFcosθ, probForMateriali, sample::materiali, sample::light (with its
    shadow ray), probForLight, the spectrum lookup and addHeroλ of the
    restatement equal the reference's (oracle/_ref) bit for bit on random
    inputs, for every material and light kind of the scene."""
    import ctypes
    fs, ref = unit_scene
    O = R.lib()
    sp = ctypes.addressof(fs.scene)
    rng = np.random.default_rng(11)
    n = 800
    ref_h = ref.h
    for m in range(fs.scene.n_materials):
        if fs.materials[m].type not in (0, 1, 2):
            continue
        lam, F, front, nz, p, i, o = _queries(ref, rng, n)
        hits = _hits(F, front, p, m)
        a = np.zeros(16, np.float32)
        b = np.zeros(16, np.float32)
        for t in range(n):
            ref.L.ref_bxdf(ref_h, m, lam[t].ctypes.data, i[t].ctypes.data, o[t].ctypes.data,
                           nz[t].ctypes.data, int(front[t]), a.ctypes.data)
            O.oracle_unit_bxdf(sp, m, lam[t].ctypes.data, i[t].ctypes.data, o[t].ctypes.data,
                               nz[t].ctypes.data, int(front[t]), b.ctypes.data)
            assert np.array_equal(_bits(a), _bits(b)), ("BxDFcosθ", m, t)
            pr = ref.L.ref_prob_for_material(ref_h, float(lam[t, 0]), ctypes.byref(hits[t]),
                                             i[t].ctypes.data, o[t].ctypes.data, 0.8)
            po = O.oracle_unit_prob_for_material(sp, float(lam[t, 0]), ctypes.byref(hits[t]),
                                                 i[t].ctypes.data, o[t].ctypes.data, 0.8)
            assert _bits(pr) == _bits(po), ("probForMateriali", m, t)
            seed = int(rng.integers(1, 2 ** 62))
            pa, pb = ctypes.c_float(), ctypes.c_float()
            da, db = np.zeros(3, np.float32), np.zeros(3, np.float32)
            ka = ref.L.ref_sample_material(ref_h, lam[t].ctypes.data, ctypes.byref(hits[t]), o[t].ctypes.data,
                                           seed, 0.8, ctypes.byref(pa), da.ctypes.data, a.ctypes.data)
            kb = O.oracle_unit_sample_material(sp, lam[t].ctypes.data, ctypes.byref(hits[t]), o[t].ctypes.data,
                                               seed, 0.8, ctypes.byref(pb), db.ctypes.data, b.ctypes.data)
            assert (ka != 0) == (kb != 0), ("sample::materiali", m, t)
            if ka:
                assert _bits(pa.value) == _bits(pb.value) and np.array_equal(_bits(da), _bits(db)), \
                    ("sample::materiali", m, t)
                assert np.array_equal(_bits(a), _bits(b)), ("sample::materiali mult", m, t)
    for li in range(fs.scene.n_lights):
        lam, F, front, nz, p, i, o = _queries(ref, rng, n)
        hits = _hits(F, front, p, 0)
        a = np.zeros(16, np.float32)
        b = np.zeros(16, np.float32)
        for t in range(n):
            seed = int(rng.integers(1, 2 ** 62))
            pa, pb = ctypes.c_float(), ctypes.c_float()
            da, db = np.zeros(3, np.float32), np.zeros(3, np.float32)
            ref.L.ref_sample_light(ref_h, li, lam[t].ctypes.data, ctypes.byref(hits[t]), seed,
                                   ctypes.byref(pa), da.ctypes.data, a.ctypes.data)
            O.oracle_unit_sample_light(sp, li, lam[t].ctypes.data, ctypes.byref(hits[t]), seed,
                                       ctypes.byref(pb), db.ctypes.data, b.ctypes.data)
            assert _bits(pa.value) == _bits(pb.value), ("sample::light prob", li, t)
            assert np.array_equal(_bits(da), _bits(db)) and np.array_equal(_bits(a), _bits(b)), \
                ("sample::light", li, t)
            ray6 = np.concatenate([p[t], i[t]]).astype(np.float32)
            assert _bits(ref.L.ref_prob_for_light(ref_h, li, ray6.ctypes.data)) == \
                _bits(O.oracle_unit_prob_for_light(sp, li, ray6.ctypes.data)), ("probForLight", li, t)
    lam, *_ = _queries(ref, rng, 200)
    for s in range(fs.scene.n_spectra):
        v = np.ascontiguousarray(fs.spectra[s], np.float32)
        a = np.zeros(16, np.float32)
        b = np.zeros(16, np.float32)
        for t in range(len(lam)):
            ref.L.ref_eval_spectrum(v.ctypes.data, lam[t].ctypes.data, a.ctypes.data)
            O.oracle_unit_spectrum(sp, s, lam[t].ctypes.data, b.ctypes.data)
            assert np.array_equal(_bits(a), _bits(b)), ("spectrum", s, t)
    nb = int(fs.scene.spec.n_bins)
    for t in range(len(lam)):
        val = rng.uniform(0, 3, 16).astype(np.float32)
        a = np.zeros(nb, np.float32)
        b = np.zeros(nb, np.float32)
        ref.L.ref_add_hero(lam[t].ctypes.data, val.ctypes.data, a.ctypes.data)
        O.oracle_unit_add_hero(sp, lam[t].ctypes.data, val.ctypes.data, b.ctypes.data)
        assert np.array_equal(_bits(a), _bits(b)), ("addHeroλ", t)


def test_instanced_scene_intersect_bit_exact(scene_dir):
    """The benchmark scene (64 instances of a 327,680-triangle displaced
    icosphere, ground, 2 quad lights): the restatement's intersect::scene
    against the reference's on camera and bounce rays and rays from inside
    overlapping object bounds."""
    from lambda_b200 import synth
    nls = synth.instanced(str(scene_dir / "instanced_full"), n_instances=64, subdiv=7, width=1920)
    sc = load_nls(nls)
    ref = refharness.RefScene(nls)
    rays = raysets.camera_rays(sc, 256, seed=31)
    rays = np.concatenate([rays, raysets.bounce_rays(ref.intersect(rays), 32),
                           raysets.overlap_origin_rays(sc, 20000, seed=33)])
    h = ref.intersect(rays)
    g = R.Oracle(flatten(sc)).intersect(rays)
    for f in ("t", "obj", "mat", "p", "n", "gn", "front"):
        assert np.array_equal(np.ascontiguousarray(h[f]).view(np.uint32),
                              np.ascontiguousarray(g[f]).view(np.uint32)), f


def test_shipped_box_fixture_reproduces_reference_rows():
    """The fixture of bin/scenes/box.nls (tests/golden/shipped_box.py) holds
    the whole scene: the restatement renders its stored reference rows bit
    for bit from the stored arrays, on the reference's own streams."""
    import ctypes
    from tests.golden import shipped_box
    fx, d = shipped_box.load()
    ref_spp, _, B = (int(x) for x in d["settings"])
    p = float(d["sample_p"][0])
    o = R.Oracle((ctypes.addressof(fx.scene), int(fx.scene.cam.width), int(fx.scene.cam.height)))
    R.lib().oracle_set_mt_arg_order(1)
    for k in (0, len(d["rows"]) // 2, len(d["rows"]) - 1):
        r = int(d["rows"][k])
        a = o.render_rows(ref_spp, B, p, r, r + 1)[0]
        assert np.array_equal(a.view(np.uint32), d["ref"][k].view(np.uint32)), k
