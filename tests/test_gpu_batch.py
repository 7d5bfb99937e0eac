"""Batched renders (lgpu_render_batch): every job's image equals the plain
render of its scene with the same settings, bit for bit — each path has its
own random stream (seed, pixel, sample) and each pixel sums its samples in
sample order, whichever kernel launch or queue position handled them."""
import os

import numpy as np
import pytest

from lambda_b200 import _lib as L
from lambda_b200 import synth
from lambda_b200.renderer import Context
from lambda_b200.scene import load_nls

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scenes(scene_dir, mixed_nls, mixed2_nls):
    inst = synth.instanced(os.path.join(str(scene_dir), "inst_batch"), n_instances=9, subdiv=3, width=48)
    small = synth.mixed(os.path.join(str(scene_dir), "mixed_batch"), width=24, seed=3)
    return [load_nls(p) for p in (mixed_nls, inst, mixed2_nls, small)]


JOBS = [
    dict(scene=0, spp=8, max_scatterings=6, sample_p=0.8, seed=1),
    dict(scene=1, spp=3, max_scatterings=12, sample_p=0.8, seed=2),
    dict(scene=2, spp=5, max_scatterings=4, sample_p=0.5, seed=3),
    dict(scene=1, spp=16, max_scatterings=2, sample_p=0.9, seed=4, spp_offset=7),
    dict(scene=3, spp=1, max_scatterings=8, sample_p=0.8, seed=5),
    dict(scene=0, spp=2, max_scatterings=6, sample_p=0.8, seed=1, flags=L.FLAG_REFERENCE_ORDER),
]


def plain(scenes, jobs):
    ctx = Context()
    out = []
    for j in jobs:
        ctx.upload(scenes[j["scene"]])
        out.append(ctx.render(j["spp"], j["max_scatterings"], j["sample_p"], seed=j["seed"],
                              flags=j.get("flags", 0), spp_offset=j.get("spp_offset", 0)))
    return out


def test_batch_equals_plain_renders(scenes):
    ref = plain(scenes, JOBS)
    ctx = Context()
    ctx.upload_many(scenes)
    imgs = ctx.render_batch(JOBS)
    st = ctx.stats()
    for k, (a, b) in enumerate(zip(imgs, ref)):
        assert a.shape == b.shape
        assert np.all(np.isfinite(a))
        assert np.array_equal(a, b), (k, np.abs(a - b).max())
    assert st["paths"] == sum(int(np.prod(ctx.slot_size(j["scene"]))) * j["spp"] for j in JOBS)
    assert st["device_checks"] == 0


def test_batch_repeatable_and_single_job(scenes):
    ctx = Context()
    ctx.upload_many(scenes)
    a = ctx.render_batch(JOBS[:3])
    b = ctx.render_batch(JOBS[:3])
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    one = ctx.render_batch(JOBS[1:2])[0]
    assert np.array_equal(one, a[1])


def test_batch_device_outputs(scenes):
    import torch
    ctx = Context()
    ctx.upload_many(scenes)
    ref = ctx.render_batch(JOBS)
    outs = [torch.empty(int(np.prod(ctx.slot_size(j["scene"]))) * 3, dtype=torch.float32, device="cuda")
            for j in JOBS]
    ctx.render_batch_device(JOBS, [o.data_ptr() for o in outs])
    torch.cuda.synchronize()
    for o, r in zip(outs, ref):
        assert np.array_equal(o.cpu().numpy().reshape(r.shape), r)


def test_batch_rejects_bad_jobs(scenes):
    ctx = Context()
    ctx.upload_many(scenes[:2])
    with pytest.raises(L.LgpuError):
        ctx.render_batch([dict(scene=2, spp=1, max_scatterings=1, sample_p=0.8)])
    with pytest.raises(L.LgpuError):
        ctx.render_batch([dict(scene=0, spp=0, max_scatterings=1, sample_p=0.8),
                          dict(scene=1, spp=1, max_scatterings=1, sample_p=0.8)])


def test_image_independent_of_launch_shape(scenes):
    """Queue depth, shading block size, trace occupancy and graph replay
    change only the schedule: images are bit-identical."""
    ctx = Context()
    ctx.upload_many(scenes)
    ref = ctx.render_batch(JOBS[:4])
    plain = Context()
    plain.upload(scenes[1])
    p_ref = plain.render(JOBS[1]["spp"], JOBS[1]["max_scatterings"], JOBS[1]["sample_p"], seed=JOBS[1]["seed"])
    for shape in (dict(queue_cap=4096), dict(shade_block=64), dict(shade_block=128), dict(trace_per_sm=3),
                  dict(graphs=0),
                  dict(queue_cap=1 << 22, shade_block=96, graphs=1)):
        ctx.set_wave_config(**shape)
        got = ctx.render_batch(JOBS[:4])
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), shape
        plain.set_wave_config(**shape)
        p = plain.render(JOBS[1]["spp"], JOBS[1]["max_scatterings"], JOBS[1]["sample_p"], seed=JOBS[1]["seed"])
        assert np.array_equal(p, p_ref), shape


def test_megakernel_split_and_autotune(scenes):
    ctx = Context()
    ctx.upload_many(scenes)
    ref = ctx.render_batch(JOBS)
    # the smallest jobs on the megakernel: same estimator and random
    # streams, different arithmetic order, so statistically equal images
    ctx.set_wave_config(mega_items=48 * 48 * 4)
    got = ctx.render_batch(JOBS)
    for a, b in zip(got, ref):
        assert a.shape == b.shape and np.all(np.isfinite(a))
        assert abs(float(a.mean()) - float(b.mean())) <= 0.05 * abs(float(b.mean())) + 1e-6
    cfg = ctx.autotune_batch(JOBS, spp_divisor=2)
    assert cfg == ctx.wave_config()
    ctx.set_wave_config(mega_items=0)
    again = ctx.render_batch(JOBS)
    for a, b in zip(again, ref):
        assert np.array_equal(a, b)


def test_tile_jobs_compose_the_frame(scenes):
    """Jobs covering rectangles of one frame (uneven split) give exactly the
    pixels of the whole-frame render."""
    ctx = Context()
    ctx.upload_many(scenes)
    w, h = ctx.slot_size(1)
    base = dict(scene=1, spp=4, max_scatterings=6, sample_p=0.8, seed=9)
    full = ctx.render_batch([base, JOBS[0]])[0]
    xs, ys = [0, w // 3, w], [0, h // 2 + 1, h]
    tiles = [dict(base, rect=(xs[a], ys[b], xs[a + 1] - xs[a], ys[b + 1] - ys[b]))
             for a in range(2) for b in range(2)]
    imgs = ctx.render_batch(tiles)
    got = np.zeros_like(full)
    for t, im in zip(tiles, imgs):
        x0, y0, tw, th = t["rect"]
        got[y0:y0 + th, x0:x0 + tw] = im[y0:y0 + th, x0:x0 + tw]
    assert np.array_equal(got, full)
    with pytest.raises(L.LgpuError):
        ctx.render_batch([dict(base, rect=(w - 2, 0, 4, 4)), JOBS[0]])
