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


@pytest.mark.parametrize("which", ["mixed_nls", "mixed2_nls", "box_nls"])
def test_render_bit_exact_with_reference_stream(which, request):
    nls = request.getfixturevalue(which)
    sc = load_nls(nls)
    ref = refharness.RefScene(nls)
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
