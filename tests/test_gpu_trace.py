"""Closest-hit parity: lgpu_trace_closest against the reference's
intersect::scene (cg.hpp:1469-1489) on identical ray sets.

With LGPU_FLAG_REFERENCE_ORDER the device visits objects and BVH children in
the reference's order, so every field is required to be bit-identical: hit
distance, object, material, world hit point, shading normal, geometric
normal, front flag.  With the instance-level BVH (default) the objects are
visited in another order and each mesh through its surface-area-heuristic
traversal tree, so at exactly equal distances (ties: two objects, or two
faces of a mesh sharing the edge the ray hits) another object or face may be
reported; the distance itself must still be bit-identical on every ray, and
every other ray identical in every field.  Faces come from the oracle's
restatement, which records them (the reference's harness does not).
"""
import numpy as np
import pytest

from lambda_b200 import _lib as L
from lambda_b200.renderer import Context
from lambda_b200.scene import FlatScene, load_nls
from oracle import refharness
from tests import raysets

pytestmark = pytest.mark.gpu

MISS = np.uint32(0xFFFFFFFF)


def _rays(sc, ref):
    cam = raysets.camera_rays(sc, 96, seed=3)
    h = ref.intersect(cam)
    bounce = raysets.bounce_rays(h, seed=4)
    h2 = ref.intersect(bounce)
    bounce2 = raysets.bounce_rays(h2, seed=5)
    rnd = raysets.random_rays([-4, -4, 0.01], [4, 4, 4], 20000, seed=6)
    return np.concatenate([cam, bounce, bounce2, rnd])


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _assert_identical(g, r, fields=("t", "obj", "mat", "p", "n", "gn", "front")):
    for f in fields:
        bad = np.nonzero(np.any((_bits(g[f]) != _bits(r[f])).reshape(len(g), -1), axis=1))[0]
        assert bad.size == 0, f"field {f}: {bad.size} of {len(g)} rays differ, e.g. ray {bad[:5]}"


@pytest.mark.parametrize("which", ["mixed_nls", "mixed2_nls", "box_nls"])
def test_closest_hit_reference_order_bit_exact(which, request):
    nls = request.getfixturevalue(which)
    sc = load_nls(nls)
    ref = refharness.RefScene(nls)
    rays = _rays(sc, ref)
    ctx = Context()
    ctx.upload(sc)
    g = ctx.trace(rays, flags=L.FLAG_REFERENCE_ORDER)
    r = ref.intersect(rays)
    assert (r["obj"] != MISS).sum() > len(rays) // 4
    _assert_identical(g, r)
    assert ctx.stats()["device_checks"] == 0


@pytest.mark.parametrize("which", ["mixed_nls", "box_nls"])
def test_closest_hit_instance_bvh(which, request):
    nls = request.getfixturevalue(which)
    sc = load_nls(nls)
    ref = refharness.RefScene(nls)
    rays = _rays(sc, ref)
    ctx = Context()
    ctx.upload(sc)
    g = ctx.trace(rays)
    r = ref.intersect(rays)
    assert np.array_equal(_bits(g["t"]), _bits(r["t"]))
    from oracle import restatement
    o = restatement.Oracle(sc).intersect(rays)
    assert np.array_equal(_bits(o["t"]), _bits(r["t"]))
    diff = (g["obj"] != r["obj"]) | (g["face"] != o["face"])
    # only ties may resolve to another object or face; everything else is identical
    same = ~diff
    _assert_identical(g[same], r[same])
    assert diff.sum() <= max(1, len(rays) // 10000)


def test_many_objects_instance_bvh(scene_dir):
    """4,160 objects (the inverse-rendering scene: one quad per albedo and
    per thickness tile).  Its surface-area-heuristic instance BVH needs more
    entries than the traversal's instance stack holds, so the upload builds
    that level with the reference's split rule instead; distances stay
    bit-identical to intersect::scene."""
    from lambda_b200 import synth
    alb = np.full((64, synth.ALBEDO_BINS), 0.5)
    th = np.full((64, 64), 400.0)
    nls = synth.diff_scene(str(scene_dir / "diff64"), alb, th, width=64)
    sc = load_nls(nls)
    ref = refharness.RefScene(nls)
    rays = _rays(sc, ref)
    r = ref.intersect(rays)
    assert (r["obj"] != MISS).sum() > len(rays) // 4
    ctx = Context()
    ctx.upload(sc)
    g = ctx.trace(rays)
    assert np.array_equal(_bits(g["t"]), _bits(r["t"]))
    assert ctx.stats()["device_checks"] == 0
    ctx.close()


def test_trace_empty_and_miss(mixed_nls):
    sc = load_nls(mixed_nls)
    ctx = Context()
    ctx.upload(sc)
    assert len(ctx.trace(np.zeros((0, 6), np.float32))) == 0
    # a ray pointing away from everything misses: t = FLT_MAX, obj = UINT32_MAX
    g = ctx.trace(np.array([[0, 0, 50, 0, 0, 1]], np.float32))
    assert g["obj"][0] == MISS and g["t"][0] == np.finfo(np.float32).max


def test_face_ids_consistent(mixed_nls):
    """The reported face of a trimesh hit reproduces the hit distance under
    the reference's triangle test restated in the C oracle."""
    from oracle import restatement
    sc = load_nls(mixed_nls)
    ref = refharness.RefScene(mixed_nls)
    rays = _rays(sc, ref)
    ctx = Context()
    ctx.upload(sc)
    g = ctx.trace(rays, flags=L.FLAG_REFERENCE_ORDER)
    o = restatement.Oracle(sc).intersect(rays)
    assert np.array_equal(g["face"], o["face"])
    assert np.array_equal(_bits(g["t"]), _bits(o["t"]))


# ---- the benchmark's own scenes, >= 10^6 rays -------------------------------------

def _large_ray_sets(sc, ref, cam_n, rnd_lo, rnd_hi, n_rnd, n_overlap):
    """Camera rays on a jittered grid, two bounce generations from the
    reference's own hits, random rays, rays from inside overlapping object
    bounds; and the shadow rays sample::light casts from every hit of the
    camera and bounce generations."""
    cam = raysets.camera_rays(sc, cam_n, seed=21)
    h0 = ref.intersect(cam)
    b1 = raysets.bounce_rays(h0, seed=22)
    h1 = ref.intersect(b1)
    b2 = raysets.bounce_rays(h1, seed=23)
    h2 = ref.intersect(b2)
    rnd = raysets.random_rays(rnd_lo, rnd_hi, n_rnd, seed=24)
    ovl = raysets.overlap_origin_rays(sc, n_overlap, seed=25)
    closest = np.concatenate([cam, b1, b2, rnd, ovl])
    hits = np.concatenate([h0, h1, h2])
    shadow = raysets.light_shadow_rays(sc, hits, seed=26)
    return closest, shadow


def _check_large(nls, cam_n, rnd_lo, rnd_hi, n_rnd, n_overlap, expect_deep):
    sc = load_nls(nls)
    ref = refharness.RefScene(nls)
    rays, (srays, tmax, skip) = _large_ray_sets(sc, ref, cam_n, rnd_lo, rnd_hi, n_rnd, n_overlap)
    assert len(rays) + len(srays) >= 1_000_000
    r = ref.intersect(rays)
    assert (r["obj"] != MISS).sum() > len(rays) // 2
    ctx = Context()
    ctx.upload(sc)
    report = {"closest_rays": len(rays), "shadow_rays": len(srays)}

    # reference order: every field of every ray bit-identical
    g = ctx.trace(rays, flags=L.FLAG_REFERENCE_ORDER)
    _assert_identical(g, r)
    assert ctx.stats()["device_checks"] == 0

    # instance BVH (the renders' default traversal): distances bit-identical
    # on every ray; another object only on an exact tie of distances
    g = ctx.trace(rays)
    st = ctx.stats()
    assert st["device_checks"] == 0
    assert np.array_equal(_bits(g["t"]), _bits(r["t"]))
    from oracle import restatement
    o = restatement.Oracle(sc).intersect(rays)
    # the restatement is pinned to the reference's distances
    assert np.array_equal(_bits(o["t"]), _bits(r["t"]))
    tie = (g["obj"] != r["obj"]) | (g["face"] != o["face"])
    _assert_identical(g[~tie], r[~tie])
    report["ties"] = int(tie.sum())
    assert tie.sum() <= max(1, len(rays) // 100000)
    report["order_rays"] = st["order_rays"]
    report["local_stack"] = st["local_stack"]
    # rays whose answer depends on the reference's object order went through
    # the linear-loop fallback, and deep BVHs spilled the traversal stack
    assert st["order_rays"] > 0
    if expect_deep:
        assert st["local_stack"] == 1

    # the reference-tree traversal of the same rays (the scene kept without
    # traversal trees): also bit-exact in distance
    flat = FlatScene(sc)
    flat.scene.flags |= L.SCENE_REFERENCE_BVH
    ctx.upload(flat)
    g2 = ctx.trace(rays)
    assert np.array_equal(_bits(g2["t"]), _bits(r["t"]))
    assert ctx.stats()["device_checks"] == 0
    ctx.upload(sc)

    # shadow rays: the reference's boolean on every ray, in both orders
    occ = ref.occluded(srays, tmax, skip)
    assert 0 < occ.sum() < len(occ)
    for flags in (0, L.FLAG_REFERENCE_ORDER):
        a = ctx.trace_any(srays, tmax, skip, flags=flags)
        bad = np.nonzero(a != occ)[0]
        assert bad.size == 0, f"flags {flags}: {bad.size} of {len(occ)} shadow rays differ, e.g. {bad[:5]}"
        assert ctx.stats()["device_checks"] == 0
    report["occluded"] = int(occ.sum())
    print(report)
    ctx.close()


def test_instanced_scene_million_rays(scene_dir):
    """The benchmark scene (64 instances of a 327,680-triangle displaced
    icosphere, ground, 2 quad lights) against intersect::scene."""
    from lambda_b200 import synth
    nls = synth.instanced(str(scene_dir / "instanced_full"), n_instances=64, subdiv=7, width=1920)
    _check_large(nls, cam_n=640, rnd_lo=[-5, -5, -0.5], rnd_hi=[5, 5, 2.5], n_rnd=120000, n_overlap=60000,
                 expect_deep=True)


def test_box_room_million_rays(scene_dir):
    """The 256x256 box room against intersect::scene."""
    from lambda_b200 import synth
    nls = synth.box_room(str(scene_dir / "box256"), width=256)
    _check_large(nls, cam_n=512, rnd_lo=[0.01, 0.01, 0.01], rnd_hi=[0.99, 0.99, 0.99], n_rnd=300000,
                 n_overlap=40000, expect_deep=False)


def test_trace_any_edges(mixed_nls):
    """Shadow-ray queries: empty input, a skipped object, a distance bound
    short of every object."""
    sc = load_nls(mixed_nls)
    ref = refharness.RefScene(mixed_nls)
    ctx = Context()
    ctx.upload(sc)
    assert len(ctx.trace_any(np.zeros((0, 6), np.float32), [], [])) == 0
    rays = _rays(sc, ref)
    for tmax, skip in ((np.float32(1e30), MISS), (np.float32(1e-3), MISS), (np.float32(1e30), np.uint32(0))):
        occ = ref.occluded(rays, np.full(len(rays), tmax, np.float32), np.full(len(rays), skip, np.uint32))
        for flags in (0, L.FLAG_REFERENCE_ORDER):
            assert np.array_equal(ctx.trace_any(rays, tmax, skip, flags=flags), occ)
