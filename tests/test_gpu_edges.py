"""Edge cases of the device renderer: ragged frame sizes (7 x 6), one sample and no
scattering, queue capacities at and around the work size, a scene without
objects (alone and in a batch), degenerate rays."""
import json
import os

import numpy as np
import pytest

from lambda_b200 import _lib as L
from lambda_b200 import synth
from lambda_b200.renderer import Context
from lambda_b200.scene import load_nls

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tiny(scene_dir):
    return load_nls(synth.mixed(os.path.join(str(scene_dir), "mixed_tiny"), width=7))


@pytest.fixture(scope="module")
def empty_scene(scene_dir):
    """A camera and a point light, no objects (the reference renders it
    black: no hit, no emission)."""
    d = os.path.join(str(scene_dir), "empty")
    os.makedirs(d, exist_ok=True)
    scene = {"camera": {"pos": [0, -5, 1], "look_at": [0, 0, 0], "up": [0, 0, 1], "fov": 45, "ar": 1.0,
                        "width": 24},
             "materials": [{"name": "m", "type": "lambertian", "albedo": {"val": 0.5}}],
             "objects": [],
             "lights": [{"name": "bulb", "type": "point", "radiant_intensity": {"val": 3.0}, "pos": [0, 0, 3]}]}
    p = os.path.join(d, "scene.nls")
    with open(p, "w") as f:
        json.dump(scene, f)
    return load_nls(p)


def test_ragged_frame_one_sample(tiny):
    ctx = Context()
    ctx.upload(tiny)
    w, h = ctx.size
    assert w == 7 and h < 8
    a = ctx.render(1, 0, 0.8, seed=1)
    b = ctx.render(1, 0, 0.8, seed=1)
    assert a.shape == (h, 7, 3) and np.all(np.isfinite(a)) and np.array_equal(a, b)
    c = ctx.render(3, 5, 0.8, seed=1)
    assert np.all(np.isfinite(c))


def test_queue_capacity_edges(mixed_nls):
    sc = load_nls(mixed_nls)
    ctx = Context()
    ctx.upload(sc)
    w, h = ctx.size
    ref = {spp: ctx.render(spp, 6, 0.8, seed=4) for spp in (1, 2, 3)}
    # queues of exactly one sample's work, one path less, and one more
    for cap in (w * h, w * h - 1, w * h + 1, 1024):
        ctx.set_wave_config(queue_cap=cap)
        for spp, img in ref.items():
            assert np.array_equal(ctx.render(spp, 6, 0.8, seed=4), img), (cap, spp)


def test_scene_without_objects(empty_scene, tiny):
    ctx = Context()
    ctx.upload(empty_scene)
    img = ctx.render(4, 4, 0.8, seed=2)
    assert np.all(img == 0)
    hits = ctx.trace(np.array([[0, -5, 1, 0, 1, -0.2], [0, 0, 0, 0, 0, 1]], np.float32))
    assert np.all(hits["obj"] == 0xFFFFFFFF)
    # in a batch, beside a scene with objects (the instance-BVH kernels)
    ctx.upload_many([empty_scene, tiny])
    imgs = ctx.render_batch([dict(scene=0, spp=2, max_scatterings=3, sample_p=0.8, seed=1),
                             dict(scene=1, spp=2, max_scatterings=3, sample_p=0.8, seed=1)])
    assert np.all(imgs[0] == 0) and np.all(np.isfinite(imgs[1]))


def test_degenerate_rays(mixed_nls):
    ctx = Context()
    ctx.upload(load_nls(mixed_nls))
    rays = np.array([[0, -6, 2.2, 0, 0, 0],            # zero direction
                     [0, -6, 2.2, 0, 1, 0],            # axis-aligned
                     [1e6, 1e6, 1e6, -1, -1, -1],      # far away, pointing back
                     [0, 0, 0.5, 0, 0, -1]], np.float32)
    h = ctx.trace(rays)
    assert len(h) == 4
    assert np.all(np.isfinite(h["t"][h["obj"] != 0xFFFFFFFF]))


def _upload(ctx, flat, host_layout):
    flat.scene.flags = L.SCENE_HOST_LAYOUT if host_layout else 0
    try:
        return ctx._lib.lgpu_upload_scene(ctx.h, flat.ptr())
    finally:
        flat.scene.flags = 0


def test_device_layout_equals_host_layout(mixed_nls, scene_dir):
    """Meshes laid out on the device at upload (the default) and on the host
    (LGPU_SCENE_HOST_LAYOUT) give bit-identical traces and renders, on the
    mixed scene and on an instanced scene of several meshes."""
    import os
    from lambda_b200 import synth
    from lambda_b200.scene import FlatScene
    from tests import raysets
    inst = synth.instanced(os.path.join(str(scene_dir), "layout_inst"), n_instances=9, subdiv=4, width=48)
    for nls in (mixed_nls, inst):
        sc = load_nls(nls)
        flat = FlatScene(sc)
        rays = np.concatenate([raysets.camera_rays(sc, 64, seed=1),
                               raysets.random_rays([-3, -3, 0.01], [3, 3, 3], 20000, seed=2)])
        out = []
        for host in (False, True):
            ctx = Context()
            assert _upload(ctx, flat, host) == L.OK
            ctx.flat = flat
            h = ctx.trace(rays)
            img = ctx.render(8, 8, 0.8, seed=4)
            out.append((h, img, ctx.stats()["upload_bytes"]))
            ctx.close()
        (h0, i0, b0), (h1, i1, b1) = out
        assert np.array_equal(h0.view(np.uint8), h1.view(np.uint8))
        assert np.array_equal(i0.view(np.uint32), i1.view(np.uint32))
        assert b0 > 0 and b1 > 0


def test_device_layout_rejects_bad_indices(mixed_nls):
    """An out-of-range vertex or BVH primitive index fails the upload with
    the mesh named, in both layouts, without the device reading it."""
    from lambda_b200.scene import FlatScene
    sc = load_nls(mixed_nls)
    m = next(mm for mm in sc.meshes if mm.F.shape[0] > 4)
    mi = sc.meshes.index(m)
    for field, bad, msg in (("F", lambda a: a.__setitem__((3, 1), 10 ** 7), "face index out of range"),
                            ("prim_idxs", lambda a: a.__setitem__(2, 10 ** 7), "primitive index out of range")):
        arr = getattr(m, field)
        saved = arr.copy()
        bad(arr)
        try:
            flat = FlatScene(sc)
            for host in (False, True):
                ctx = Context()
                rc = _upload(ctx, flat, host)
                assert rc == L.ERR_INVALID_ARGUMENT, (field, host, rc)
                err = ctx._lib.lgpu_last_error(ctx.h).decode()
                assert msg in err and ("mesh %d" % mi) in err, err
                ctx.close()
        finally:
            arr[...] = saved


def test_upload_builds_missing_bvh(mixed_nls):
    """Meshes passed without their BVH (nodes, bbs, prim_idxs NULL) get the
    tree bvh::build would make, built on the device at upload: traces and
    renders are bit-identical to those of the scene with the reference's
    trees."""
    from lambda_b200.scene import FlatScene
    from tests import raysets
    sc = load_nls(mixed_nls)
    rays = np.concatenate([raysets.camera_rays(sc, 48, seed=7),
                           raysets.random_rays([-3, -3, 0.01], [3, 3, 3], 10000, seed=8)])
    outs = []
    for strip in (False, True):
        flat = FlatScene(sc)
        if strip:
            for k in range(int(flat.scene.n_meshes)):
                m = flat.meshes[k]
                m.nodes, m.bbs, m.prim_idxs = None, None, None
                m.n_nodes = m.n_bbs = m.n_prim_idxs = 0
        ctx = Context()
        ctx.upload(flat)
        outs.append((ctx.trace(rays), ctx.render(8, 8, 0.8, seed=3)))
        ctx.close()
    assert np.array_equal(outs[0][0].view(np.uint8), outs[1][0].view(np.uint8))
    assert np.array_equal(outs[0][1].view(np.uint32), outs[1][1].view(np.uint32))
