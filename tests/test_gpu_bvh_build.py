"""The device BVH builder (lgpu_build_bvh_device) against the host
restatement of bvh::build (lgpu_build_bvh, itself pinned to the reference's
trees by the loader tests): node records, child boxes and primitive order
bit-identical, on meshes of every size and on the builder's corner cases —
a bin that takes every triangle (the redistribution into 8 chunks), flat and
point-like triangles, ties between +0 and -0 in the boxes."""
import time

import numpy as np
import pytest

from lambda_b200 import synth
from lambda_b200.renderer import Context

pytestmark = pytest.mark.gpu


def _with_dummy(V):
    return np.concatenate([np.zeros((1, 3), np.float32), np.asarray(V, np.float32)])


def _soup(n, seed, spread=4.0):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 1, 3))
    V = (c + rng.normal(scale=0.05, size=(n, 3, 3))).reshape(-1, 3)
    F = np.arange(1, 3 * n + 1, dtype=np.uint32).reshape(n, 3)
    return _with_dummy(V), F


def _mesh_cases():
    cases = {}
    for sd in (3, 5, 7):
        V, N, F = synth.displaced_icosphere(sd, 11, amp=0.06)
        cases["icosphere%d" % sd] = (_with_dummy(V), np.asarray(F, np.uint32)[:, :3] + 1)
    V, N, F = synth.displaced_uv_sphere(3)
    cases["uv64k"] = (_with_dummy(V), np.asarray(F, np.uint32)[:, :3] + 1)
    for n in (1, 2, 4, 5, 9, 17, 40, 1000):
        cases["soup%d" % n] = _soup(n, n)
    cases["soup100k"] = _soup(100000, 7)
    # every triangle the same: each split puts all of them in one bin
    t = np.array([[0.1, 0.2, 0.3], [0.5, 0.2, 0.3], [0.1, 0.7, 0.3]], np.float32)
    cases["identical"] = (_with_dummy(np.tile(t, (300, 1))), np.arange(1, 901, dtype=np.uint32).reshape(300, 3))
    # point-like triangles at one point: zero extents, undefined bins
    cases["points"] = (_with_dummy(np.full((60, 3), 0.25, np.float32)),
                       np.arange(1, 61, dtype=np.uint32).reshape(20, 3))
    # flat in z, and +0 / -0 minima on every axis
    rng = np.random.default_rng(3)
    V = rng.uniform(0, 1, (3000, 3)).astype(np.float32)
    V[:, 2] = 0.0
    V[rng.random(3000) < 0.3, 0] = 0.0
    neg = rng.random(3000) < 0.5
    V[neg & (V[:, 0] == 0), 0] = -0.0
    V[neg, 2] = -0.0
    cases["signed_zeros"] = (_with_dummy(V), np.arange(1, 3001, dtype=np.uint32).reshape(1000, 3))
    # faces with more than 3 words per face (the loader's 6: V then N indices)
    V, F = _soup(500, 9)
    cases["stride6"] = (V, np.concatenate([F, F], axis=1))
    return cases


@pytest.fixture(scope="module")
def ctx():
    c = Context()
    yield c
    c.close()


@pytest.mark.parametrize("name", list(_mesh_cases().keys()))
def test_device_build_is_bit_identical(ctx, name):
    V, F = _mesh_cases()[name]
    t0 = time.perf_counter()
    h = ctx.build_bvh(V, F, device=False)
    t1 = time.perf_counter()
    d = ctx.build_bvh(V, F, device=True)
    t2 = time.perf_counter()
    assert np.array_equal(d[0], h[0]), "nodes"
    assert np.array_equal(d[1].view(np.uint32), h[1].view(np.uint32)), "child boxes"
    assert np.array_equal(d[2], h[2]), "primitive order"
    assert sorted(d[2].tolist()) == list(range(F.shape[0]))
    print(f"{name}: {F.shape[0]} faces, {len(h[0]) // 2} nodes; host {1e3 * (t1 - t0):.1f} ms, "
          f"device {1e3 * (t2 - t1):.1f} ms")


def test_device_build_rejects_bad_faces(ctx):
    from lambda_b200 import _lib as L
    V, F = _soup(10, 1)
    F = F.copy()
    F[3, 1] = V.shape[0]
    with pytest.raises(L.LgpuError):
        ctx.build_bvh(V, F, device=True)
    V, F = _soup(10, 2)
    V[5, 1] = np.nan
    with pytest.raises(L.LgpuError):
        ctx.build_bvh(V, F, device=True)
