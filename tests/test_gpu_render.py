"""Image parity of the device renderer against the reference renderer.

The device and the reference use different random streams (counter-based
PCG32 per path vs one mt19937 per pixel), so images are compared
statistically: both are measured against an FP64-accumulated high-spp image
of the reference (the oracle, on streams disjoint from both) at matched spp.
The error of a render is heavy-tailed (a few firefly pixels of specular
paths can carry most of its MSE and change it tenfold between seeds, even
as a median over 16 renders), so the noise is compared through the
distribution of per-pixel errors instead: |img - oracle| / RMS(oracle) per
channel, pooled over N_RENDERS independent renders per side, at its median
and 90th percentile.  These are stable to 1-2 % between seed sets, and the
device's must equal the reference's within QUANT_TOL (two-sided).  The
median-of-renders rel MSE (sum((img - oracle)^2) / sum(oracle^2)) is
reported beside them.

Bias: every pixel draws its own streams on both sides, so the per-pixel
differences between a high-spp device image and the oracle are independent;
their mean over the image, divided by its standard error, must stay within
T_MAX per channel (a few standard errors: no systematic difference between
the estimators at the precision the sample size resolves).
"""
import numpy as np
import pytest

from lambda_b200 import _lib as L
from lambda_b200.renderer import Context
from lambda_b200.scene import load_nls
from oracle import refharness

pytestmark = pytest.mark.gpu

ORACLE_SPP = 1024
QUANT_TOL = 0.05   # |device / reference - 1| of the pooled error quantiles, per channel
T_MAX = 4.5        # |mean per-pixel difference| / its standard error, per channel
N_RENDERS = 16     # independent renders per side


def rel_mse(img, oracle):
    return np.sum((img - oracle) ** 2, axis=(0, 1)) / np.sum(oracle ** 2, axis=(0, 1))


def bias_t(img, oracle):
    """Per channel: mean of the per-pixel differences over its standard
    error, and the ratio of the image means."""
    d = (np.asarray(img, np.float64) - oracle).reshape(-1, 3)
    se = d.std(axis=0, ddof=1) / np.sqrt(d.shape[0])
    ratio = np.asarray(img, np.float64).reshape(-1, 3).mean(0) / np.asarray(oracle).reshape(-1, 3).mean(0)
    return d.mean(axis=0) / np.maximum(se, 1e-30), ratio


def error_stats(imgs, oracle):
    """(pooled per-pixel error quantiles [q50, q90] per channel, median rel
    MSE) of renders against the oracle."""
    oracle = np.asarray(oracle, np.float64)
    scale = np.sqrt(np.mean(oracle ** 2, axis=(0, 1)))
    e = np.abs(np.stack(imgs).astype(np.float64) - oracle).reshape(-1, 3) / scale
    return np.percentile(e, [50, 90], axis=0), np.median([rel_mse(im, oracle) for im in imgs], axis=0)


def ref_error_stats(ref, spp, B, p, oracle, n=N_RENDERS):
    """error_stats of n reference renders at spp on independent streams
    (seed bases 2*w*h, 3*w*h, ...: disjoint from the oracle's w*h)."""
    W, H = ref.width, ref.height
    return error_stats([ref.render_rows(spp, B, p, 0, H, seed_base=(2 + k) * W * H)[::-1] for k in range(n)],
                       oracle)


def _assert_matches(ctx, ref_stats_of_spp, oracle, spp_list, hi_spp, B, p, flags=0, rows=None):
    """The device's error distribution at each spp equals the reference's
    (ref_stats_of_spp(spp) = error_stats of its renders), both against the
    oracle, and no bias at hi_spp; `rows` selects image rows (top-first)
    when the oracle covers only those."""
    sel = (lambda x: x) if rows is None else (lambda x: x[rows])
    report = {}
    for spp in spp_list:
        gs = [sel(ctx.render(spp, B, p, seed=1000 + k, flags=flags)) for k in range(N_RENDERS)]
        assert all(np.all(np.isfinite(g)) for g in gs)
        q_gpu, m_gpu = error_stats(gs, oracle)
        q_ref, m_ref = ref_stats_of_spp(spp)
        r = q_gpu / q_ref
        report[spp] = {"quantile_ratio": r.round(4).tolist(), "median_mse_ratio": (m_gpu / m_ref).round(3).tolist()}
        assert np.all(np.abs(r - 1.0) <= QUANT_TOL), (spp, q_gpu, q_ref)
    g = ctx.render(hi_spp, B, p, seed=99, flags=flags)
    t, ratio = bias_t(sel(g), oracle)
    report["t"] = t.round(2).tolist()
    report["mean_ratio"] = ratio.round(5).tolist()
    print(report)
    assert np.all(np.abs(t) <= T_MAX), (t, ratio)
    assert ctx.stats()["device_checks"] == 0


@pytest.fixture(scope="module")
def small_mixed(scene_dir):
    import os
    from lambda_b200 import synth
    return synth.mixed(os.path.join(str(scene_dir), "mixed_small"), width=40)


def _fp64_oracle(ref, spp, B, p):
    """The reference's FP64-film image at spp from streams disjoint from
    its own render's (seed base w*h), row 0 at the top."""
    band = ref.render_rows(spp, B, p, 0, ref.height, fp64=True, seed_base=ref.width * ref.height)
    return band[::-1].copy()


@pytest.mark.parametrize("flags", [0, L.FLAG_REFERENCE_ORDER])
def test_render_rel_mse_matches_reference(small_mixed, flags):
    ref = refharness.RefScene(small_mixed)
    oracle = _fp64_oracle(ref, ORACLE_SPP, 8, 0.8)
    ctx = Context()
    ctx.upload(load_nls(small_mixed))
    _assert_matches(ctx, lambda spp: ref_error_stats(ref, spp, 8, 0.8, oracle), oracle, (16, 64), 4096, 8, 0.8,
                    flags)


def test_box_room_config_matches_k4_reference(scene_dir):
    """The box-room configuration (256x256, 16 spp, 8 bounces, p = 0.8, 4
    hero wavelengths over 380-780 nm in 81 bins) against the reference
    built at that spectral setting (oracle/_ref/libref_k4.so)."""
    import os
    from lambda_b200 import synth
    nls = synth.box_room(os.path.join(str(scene_dir), "box_cfg1"), width=256)
    ref = refharness.RefScene(nls, k4=True)
    assert ref.L.ref_hero_samples() == 4 and ref.L.ref_n_bins() == 81
    oracle = _fp64_oracle(ref, 512, 8, 0.8)
    ctx = Context()
    ctx.upload(load_nls(nls, refharness.spectral_config(ref.L)))
    _assert_matches(ctx, lambda spp: ref_error_stats(ref, spp, 8, 0.8, oracle), oracle, (16,), 256, 8, 0.8)


def test_depth_of_field_matches_reference(scene_dir):
    """A thin-lens camera (dof 0.2 as the reference's own published scene
    uses, focused at 2.5 units, in front of the objects 4.5-7 units away,
    which are strongly defocused): the lens branch of sample::camera
    (cg.hpp:1539)."""
    import os
    from lambda_b200 import synth
    nls = synth.mixed(os.path.join(str(scene_dir), "mixed_dof"), width=40, dof=0.2, focal=2.5)
    ref = refharness.RefScene(nls)
    oracle = _fp64_oracle(ref, ORACLE_SPP, 8, 0.8)
    ctx = Context()
    sc = load_nls(nls)
    assert abs(sc.cam.dof - 0.2) < 1e-6
    ctx.upload(sc)
    _assert_matches(ctx, lambda spp: ref_error_stats(ref, spp, 8, 0.8, oracle), oracle, (16, 64), 4096, 8, 0.8)
    # the lens matters: pinhole renders of the same scene are far further
    # from the oracle than the lens renders at the same spp
    lens = error_stats([ctx.render(256, 8, 0.8, seed=7 + k) for k in range(4)], oracle)[0][0]
    sc.cam.dof = 0.0
    ctx.upload(sc)
    pin = error_stats([ctx.render(256, 8, 0.8, seed=7 + k) for k in range(4)], oracle)[0][0]
    assert np.all(pin > 1.1 * lens), (pin, lens)


def test_shipped_box_scene_matches_reference():
    """The reference's own bin/scenes/box.nls (spheres, planes, a sphere
    light, RGB and measured spectra), from the fixture generated with the
    reference's loader and renderer (tests/golden/shipped_box.py): the
    reference's error statistics over independent renders of those rows at
    64 spp and an FP64 1024-spp oracle of the same rows."""
    from tests.golden import shipped_box
    fx, d = shipped_box.load()
    ref_spp, orc_spp, B = (int(x) for x in d["settings"])
    p = float(d["sample_p"][0])
    ctx = Context()
    L.check(ctx.h, ctx._lib.lgpu_upload_scene(ctx.h, fx.ptr()), "upload")
    ctx.flat = fx
    H = int(fx.scene.cam.height)
    rows = H - 1 - d["rows"]  # scene rows -> image rows (row 0 at the top)
    assert int(d["ref_renders"][0]) == N_RENDERS
    _assert_matches(ctx, lambda spp: (d["ref_err_quantiles"], d["ref_mse_median"]), d["oracle"].astype(np.float64),
                    (ref_spp,), 4096, B, p, rows=rows)


def test_render_deterministic(small_mixed):
    sc = load_nls(small_mixed)
    ctx = Context()
    ctx.upload(sc)
    a = ctx.render(8, 6, 0.8, seed=5)
    b = ctx.render(8, 6, 0.8, seed=5)
    c = ctx.render(8, 6, 0.8, seed=6)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)


def test_tonemap_matches_reference(small_mixed):
    ref = refharness.RefScene(small_mixed)
    img = ref.render(32, 8, 0.8)
    tm_r = np.zeros_like(img)
    b_r = np.zeros(img.shape, np.uint8)
    ref.L.ref_tonemap(img.ctypes.data, img.shape[1], img.shape[0], 0.12, tm_r.ctypes.data,
                      b_r.ctypes.data)
    ctx = Context()
    tm_g, b_g = ctx.tonemap(img, 0.12)
    # the reference sums log-luminance sequentially in float; the device sums
    # in double: tone-mapped values agree to 1e-4 relative, bytes within 1
    assert np.allclose(tm_g, tm_r, rtol=1e-4, atol=1e-6)
    assert np.max(np.abs(b_g.astype(int) - b_r.astype(int))) <= 1


@pytest.mark.parametrize("n_inst", [2, 12])
def test_kernel_timing_changes_nothing(scene_dir, n_inst):
    """FLAG_KERNEL_TIMING only adds event records and splits the work
    counters per kernel kind: the image is bit-identical and the per-kind
    counters add up to the totals."""
    import os
    from lambda_b200 import synth
    nls = synth.instanced(os.path.join(str(scene_dir), "inst_timing_%d" % n_inst),
                          n_instances=n_inst, subdiv=3, width=64)
    ctx = Context()
    ctx.upload(load_nls(nls))
    a = ctx.render(8, 8, 0.8, seed=3)
    s0 = ctx.stats()
    b = ctx.render(8, 8, 0.8, seed=3, flags=L.FLAG_KERNEL_TIMING)
    s1 = ctx.stats()
    assert np.array_equal(a, b)
    assert s0["rays"] == s1["rays"] and s0["node_tests"] == s1["node_tests"]
    assert s0["launches"] == s1["launches"] > 0
    ks = s1["kernels"]
    assert ks[0]["rays"] + ks[1]["rays"] == s1["rays"]
    assert ks[0]["node_tests"] + ks[1]["node_tests"] == s1["node_tests"]
    assert ks[0]["tri_tests"] + ks[1]["tri_tests"] == s1["tri_tests"]
    assert all(k["launches"] == ks[0]["launches"] > 0 for k in ks)
    assert all(k["ms"] > 0 for k in ks)
    assert all(k["ms"] == 0 for k in s0["kernels"])


def _overlapping_meshes(out_dir):
    """Five displaced spheres (one mesh, five instances) whose bounds
    overlap, on a quad floor: a ray leaving one sphere starts inside the
    bounds of another, which is where the reference's answer depends on its
    object order (cg.hpp:1393, 1414).  Six objects: scenes of up to four
    take every ray through the linear loop anyway."""
    import json
    import os
    from lambda_b200 import synth
    os.makedirs(out_dir, exist_ok=True)
    mesh = os.path.join(out_dir, "ico.obj")
    V, N, F = synth.displaced_icosphere(3, 5, amp=0.08)
    synth.write_indexed_obj(mesh, V, N, F)
    objs = [{"name": "floor", "type": "plane", "transform": {"scale": [6, 6, 1]}, "material": "white"}]
    for k, (x, y) in enumerate([(0.0, 0.0), (0.45, 0.3), (-0.35, 0.4), (0.3, -0.4), (-0.5, -0.3)]):
        objs.append({"name": "s%d" % k, "type": "trimesh", "material": ["white", "gloss"][k % 2],
                     "source": mesh, "transform": {"translate": [x, y, 1.0]}})
    scene = {"camera": {"pos": [0.0, -5.0, 2.5], "look_at": [0.0, 0.0, 1.0], "up": [0, 0, 1],
                        "fov": 40, "ar": 1.0, "width": 48},
             "materials": [{"name": "white", "type": "lambertian", "albedo": {"val": 0.7}},
                           {"name": "gloss", "type": "blinn", "Kd": {"val": 0.3}, "Ks": {"val": 0.5},
                            "glossiness": 32}],
             "objects": objs,
             "lights": [{"name": "sky", "type": "direction", "radiant_intensity": {"val": 1.0},
                         "dir": [0.2, 0.3, -0.9]},
                        {"name": "amb", "type": "ambient", "radiance": {"val": 0.2}}]}
    path = os.path.join(out_dir, "scene.nls")
    with open(path, "w") as f:
        json.dump(scene, f)
    return path


def test_order_dependent_rays_follow_the_reference_loop(scene_dir):
    """Rays whose closest hit depends on the reference's object order (more
    than one mesh's bounds contain their origin) are re-traced with its
    linear object loop, so the instance-BVH render equals the render that
    takes every ray through that loop (LGPU_FLAG_REFERENCE_ORDER)."""
    import os
    nls = _overlapping_meshes(os.path.join(str(scene_dir), "overlap"))
    ctx = Context()
    ctx.upload(load_nls(nls))
    a = ctx.render(8, 8, 0.8, seed=5)
    n_order = ctx.stats()["order_rays"]
    b = ctx.render(8, 8, 0.8, seed=5, flags=L.FLAG_REFERENCE_ORDER)
    assert n_order > 100, n_order
    assert ctx.stats()["order_rays"] == 0  # that render traces every ray in order
    same = np.all(a == b, axis=2).mean()
    # only rays with two objects at exactly the same distance may differ
    assert same >= 0.999, same


def test_fp64_film(small_mixed):
    """LGPU_FLAG_FP64_FILM: the same paths summed in double into an image of
    doubles, equal to the float film up to the float film's rounding;
    refused where it does not apply."""
    ctx = Context()
    ctx.upload(load_nls(small_mixed))
    a = ctx.render(64, 8, 0.8, seed=3)
    b = ctx.render(64, 8, 0.8, seed=3, flags=L.FLAG_FP64_FILM)
    assert b.dtype == np.float64 and np.all(np.isfinite(b))
    scale = np.abs(b).max()
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6 * scale)
    assert not np.array_equal(a.astype(np.float64), b)  # it is not the float film widened
    for flags in (L.FLAG_FP64_FILM | L.FLAG_MEGAKERNEL,):
        with pytest.raises(L.LgpuError) as e:
            ctx.render(4, 8, 0.8, flags=flags)
        assert e.value.code == L.ERR_UNSUPPORTED
    w, h = ctx.size
    with pytest.raises(L.LgpuError) as e:
        ctx.adjoint(4, 8, 0.8, np.zeros((h, w, 3), np.float32), flags=L.FLAG_FP64_FILM)
    assert e.value.code == L.ERR_UNSUPPORTED
