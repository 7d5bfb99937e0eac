"""Edge cases of the device renderer: ragged frame sizes (7 x 6), one sample and no
scattering, queue capacities at and around the work size, a scene without
objects (alone and in a batch), degenerate rays."""
import json
import os

import numpy as np
import pytest

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
