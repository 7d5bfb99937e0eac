"""Unit parity of the device's shading functions with the reference's own.

lgpu_probe_shading runs the device functions the render kernels use —
BxDFcosθ, probForMateriali, sample::materiali, sample::light, probForLight
and the spectrum lookup — on explicit inputs; the reference compiled from
its sources (oracle/_ref) runs its functions of the same names (cg.hpp) on
the same inputs, for every material and light kind of one scene.

Sampling gets the reference's uniform draws.  The reference draws from a
std::mt19937 seeded per query (stoch.hpp:30-47); g++ evaluates the two draws
of f(rng.flt(), rng.flt()) right to left, so the device, which takes its
draws in order, is given the pair swapped.  The shadow ray of a light sample
is traced by the reference (ref_occluded) along the device's direction.

Tolerances: neither side contracts multiply-adds, but the device uses CUDA's
powf / sincosf / cosf / logf where the reference uses libm, so values agree
to rounding, amplified by the lobe exponents (powf(x, α) with α up to 2048
turns a relative error ε of x into α·ε).  A query's error is
max_k |device - reference| / max_k |reference|; the bar is VALUE_RTOL (or
4·α ulps) for all but FLIP_FRAC of the queries (a rounding difference can
flip a branch: a direction grazing the surface, total internal reflection at
the boundary) and a median below MEDIAN_RTOL (or 2·α ulps).
"""
import ctypes
import os

import numpy as np
import pytest

from lambda_b200 import _lib as L
from lambda_b200 import synth
from lambda_b200.renderer import Context
from lambda_b200.scene import flatten, load_nls
from oracle import refharness

pytestmark = pytest.mark.gpu

VALUE_RTOL = 2e-3
MEDIAN_RTOL = 1e-5
FLIP_FRAC = 2e-3
DIR_ATOL = 1e-4
N = 4096


def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def _frames(rng, n):
    z = _unit(rng, n)
    a = np.where(np.abs(z[:, :1]) < 0.9, [[1.0, 0.0, 0.0]], [[0.0, 1.0, 0.0]])
    x = np.cross(z, a)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    y = np.cross(z, x)
    return np.concatenate([x, y, z], axis=1).astype(np.float32)


def _toward(rng, n, F, front, frac_up=0.75):
    """Directions mostly on the side of the surface the hit faces."""
    d = _unit(rng, n)
    nz = F[:, 6:9] * np.where(front, 1.0, -1.0)[:, None]
    up = rng.random(n) < frac_up
    flip = up & (np.sum(d * nz, axis=1) < 0)
    d[flip] *= -1
    return d.astype(np.float32)


@pytest.fixture(scope="module")
def unit_scene(scene_dir):
    nls = synth.mixed(os.path.join(str(scene_dir), "units"),
                      lights=("sphere", "quaddir", "point", "direction", "ambient"), width=16, seed=5)
    fs = flatten(load_nls(nls))
    ctx = Context()
    ctx.upload(fs)
    ref = refharness.RefScene(nls)
    yield fs, ctx, ref
    ctx.close()
    ref.close()


def _queries(ref, rng, n, op, index, sample_p=0.8):
    q = np.zeros(n, L.PROBE_DTYPE)
    q["op"] = op
    q["index"] = index
    seeds = rng.integers(1, 2 ** 62, n, dtype=np.uint64)
    lam = np.zeros(16, np.float32)
    for t in range(n):
        ref.L.ref_hero(int(seeds[t]), lam.ctypes.data)
        q["lambda"][t] = lam
    front = rng.random(n) < 0.8
    F = _frames(rng, n)
    q["F"] = F
    q["front"] = front
    q["p"] = rng.uniform([-2, -2, 0], [2, 2, 2], (n, 3)).astype(np.float32)
    q["o"] = _toward(rng, n, F, front)
    q["i"] = _toward(rng, n, F, front)
    q["n"] = F[:, 6:9] * np.where(front, 1.0, -1.0)[:, None]
    q["sample_p"] = sample_p
    return q, seeds


def _ref_hit(q):
    h = refharness.RefHit()
    h.z = 0.0
    h.p[:] = q["p"].tolist()
    F = q["F"].tolist()
    h.Fx[:], h.Fy[:], h.Fz[:] = F[0:3], F[3:6], F[6:9]
    h.gn[:] = F[6:9]
    h.front = int(q["front"])
    h.mat = int(q["index"])
    h.obj = 0xFFFFFFFF
    return h


def _value_errors(dev, ref):
    scale = np.abs(ref).max(axis=1)
    err = np.abs(dev - ref).max(axis=1)
    return np.where(scale > 0, err / np.maximum(scale, 1e-30), err)


def _check(err, what, alpha=0.0):
    """alpha: the lobe exponent of the material, which multiplies the
    relative error of its cosine (the sampled directions differ by an ulp
    where CUDA's and libm's powf / sincosf round differently)."""
    bad = err > max(VALUE_RTOL, 4 * alpha * 2.0 ** -24)
    assert bad.mean() <= FLIP_FRAC, (what, bad.mean(), np.sort(err)[-5:])
    med = max(MEDIAN_RTOL, 2 * alpha * 2.0 ** -24)
    assert np.median(err) <= med, (what, np.median(err), med)


def _materials(fs):
    return [k for k in range(fs.scene.n_materials)
            if fs.materials[k].type in (L.MAT_LAMBERTIAN, L.MAT_BLINN, L.MAT_THINFILM)]


def test_bxdf_matches_reference(unit_scene):
    fs, ctx, ref = unit_scene
    rng = np.random.default_rng(1)
    mats = _materials(fs)
    assert {fs.materials[k].type for k in mats} == {L.MAT_LAMBERTIAN, L.MAT_BLINN, L.MAT_THINFILM}
    for m in mats:
        q, _ = _queries(ref, rng, N, L.PROBE_BXDF, m)
        r = ctx.probe(q)
        want = np.zeros((N, 16), np.float32)
        for t in range(N):
            ref.L.ref_bxdf(ref.h, m, q["lambda"][t].ctypes.data, q["i"][t].ctypes.data,
                           q["o"][t].ctypes.data, q["n"][t].ctypes.data, int(q["front"][t]),
                           want[t].ctypes.data)
        assert np.count_nonzero(want) > N  # the queries reach the lobes
        _check(_value_errors(r["value"], want), f"BxDFcosθ material {m}", fs.materials[m].alpha)


def test_prob_for_material_matches_reference(unit_scene):
    fs, ctx, ref = unit_scene
    rng = np.random.default_rng(2)
    for m in _materials(fs):
        q, _ = _queries(ref, rng, N, L.PROBE_PROB_MATERIAL, m)
        r = ctx.probe(q)
        want = np.zeros(N, np.float32)
        for t in range(N):
            h = _ref_hit(q[t])
            want[t] = ref.L.ref_prob_for_material(ref.h, float(q["lambda"][t][0]), ctypes.byref(h),
                                                  q["i"][t].ctypes.data, q["o"][t].ctypes.data,
                                                  float(q["sample_p"][t]))
        assert np.count_nonzero(want) > N // 4
        _check(_value_errors(r["prob"][:, None], want[:, None]), f"probForMateriali material {m}",
               fs.materials[m].alpha)


def test_sample_material_matches_reference(unit_scene):
    fs, ctx, ref = unit_scene
    rng = np.random.default_rng(3)
    for m in _materials(fs):
        q, seeds = _queries(ref, rng, N, L.PROBE_SAMPLE_MATERIAL, m)
        draws = np.zeros(3, np.float32)
        for t in range(N):
            ref.L.ref_rng_flt(int(seeds[t]), 3, draws.ctypes.data)
            # the lobe draw, then f(rng.flt(), rng.flt()) evaluated right to left
            q["xi"][t][:3] = [draws[0], draws[2], draws[1]]
        r = ctx.probe(q)
        ok = np.zeros(N, bool)
        prob = np.zeros(N, np.float32)
        d = np.zeros((N, 3), np.float32)
        mult = np.zeros((N, 16), np.float32)
        for t in range(N):
            h = _ref_hit(q[t])
            pr = ctypes.c_float(0.0)
            ok[t] = ref.L.ref_sample_material(ref.h, q["lambda"][t].ctypes.data, ctypes.byref(h),
                                              q["o"][t].ctypes.data, int(seeds[t]),
                                              float(q["sample_p"][t]), ctypes.byref(pr),
                                              d[t].ctypes.data, mult[t].ctypes.data) != 0
            prob[t] = pr.value
        dev_ok = r["ok"] != 0
        assert ok.sum() > N // 4
        assert np.mean(dev_ok != ok) <= FLIP_FRAC, (m, np.mean(dev_ok != ok))
        both = dev_ok & ok
        close_dir = np.all(np.abs(r["dir"][both] - d[both]) <= DIR_ATOL, axis=1)
        assert close_dir.mean() >= 1 - FLIP_FRAC, (m, close_dir.mean())
        a = fs.materials[m].alpha
        _check(_value_errors(r["prob"][both][:, None], prob[both][:, None]), f"sample prob material {m}", a)
        _check(_value_errors(r["value"][both], mult[both]), f"sample mult material {m}", a)


def _light_draws(kind, draws):
    if kind == L.LIGHT_AMBIENT:  # f(rng.flt(), rng.flt()), right to left
        return [draws[1], draws[0]]
    return [draws[0], draws[1]]


def test_sample_light_matches_reference(unit_scene):
    fs, ctx, ref = unit_scene
    rng = np.random.default_rng(4)
    kinds = set()
    for li in range(fs.scene.n_lights):
        kind = fs.lights[li].type
        kinds.add(kind)
        q, seeds = _queries(ref, rng, N, L.PROBE_SAMPLE_LIGHT, li)
        draws = np.zeros(2, np.float32)
        for t in range(N):
            ref.L.ref_rng_flt(int(seeds[t]), 2, draws.ctypes.data)
            q["xi"][t][:2] = _light_draws(kind, draws)
        r = ctx.probe(q)
        prob = np.zeros(N, np.float32)
        d = np.zeros((N, 3), np.float32)
        mult = np.zeros((N, 16), np.float32)
        for t in range(N):
            h = _ref_hit(q[t])
            pr = ctypes.c_float(0.0)
            ref.L.ref_sample_light(ref.h, li, q["lambda"][t].ctypes.data, ctypes.byref(h), int(seeds[t]),
                                   ctypes.byref(pr), d[t].ctypes.data, mult[t].ctypes.data)
            prob[t] = pr.value
        assert np.all(np.abs(r["dir"] - d) <= DIR_ATOL), li
        _check(_value_errors(r["prob"][:, None], prob[:, None]), f"light {li} prob")
        # the device leaves visibility to the shadow ray it describes
        has_ray = r["tmax"] >= 0
        vis = np.ones(N, bool)
        if has_ray.any():
            rays = np.concatenate([q["p"], r["dir"]], axis=1)[has_ray]
            vis[has_ray] = ~ref.occluded(rays, r["tmax"][has_ray], r["skip"][has_ray])
        dev = r["value"] * vis[:, None]
        _check(_value_errors(dev, mult), f"light {li} mult")
    assert kinds == {L.LIGHT_SPHERE, L.LIGHT_QUADDIR, L.LIGHT_POINT, L.LIGHT_DIR, L.LIGHT_AMBIENT}


def test_prob_for_light_matches_reference(unit_scene):
    fs, ctx, ref = unit_scene
    rng = np.random.default_rng(5)
    for li in range(fs.scene.n_lights):
        lt = fs.lights[li]
        q, _ = _queries(ref, rng, N, L.PROBE_PROB_LIGHT, li)
        # aim half of the rays at the light (its transform's origin)
        c = np.array([lt.T.M[3], lt.T.M[7], lt.T.M[11]], np.float32)
        aim = c[None, :] + rng.normal(scale=0.4, size=(N, 3)) - q["p"]
        aim /= np.linalg.norm(aim, axis=1, keepdims=True)
        half = rng.random(N) < 0.5
        q["i"][half] = aim[half].astype(np.float32)
        r = ctx.probe(q)
        want = np.zeros(N, np.float32)
        for t in range(N):
            ray6 = np.concatenate([q["p"][t], q["i"][t]]).astype(np.float32)
            want[t] = ref.L.ref_prob_for_light(ref.h, li, ray6.ctypes.data)
        if lt.type in (L.LIGHT_SPHERE, L.LIGHT_QUADDIR):
            assert np.count_nonzero(want) > N // 8, li
        _check(_value_errors(r["prob"][:, None], want[:, None]), f"probForLight light {li}")


def test_spectrum_lookup_matches_reference(unit_scene):
    fs, ctx, ref = unit_scene
    rng = np.random.default_rng(6)
    n_spec = fs.spectra.shape[0]
    for s in range(n_spec):
        q, _ = _queries(ref, rng, 512, L.PROBE_SPECTRUM, s)
        r = ctx.probe(q)
        want = np.zeros((512, 16), np.float32)
        v = np.ascontiguousarray(fs.spectra[s], np.float32)
        for t in range(512):
            ref.L.ref_eval_spectrum(v.ctypes.data, q["lambda"][t].ctypes.data, want[t].ctypes.data)
        err = _value_errors(r["value"], want)
        assert err.max() <= 1e-6, (s, err.max())


def test_probe_rejects_bad_queries(unit_scene):
    fs, ctx, ref = unit_scene
    q = np.zeros(2, L.PROBE_DTYPE)
    q["op"] = L.PROBE_BXDF
    q["index"][1] = fs.scene.n_materials
    with pytest.raises(L.LgpuError):
        ctx.probe(q)
    q["index"][1] = 0
    q["op"][0] = 99
    with pytest.raises(L.LgpuError):
        ctx.probe(q)
