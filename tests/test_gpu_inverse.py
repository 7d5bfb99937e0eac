"""The torch.autograd.Function over the renderer and its adjoint, and the
inverse-rendering harness on a small diff_scene."""
import numpy as np
import pytest

from lambda_b200 import inverse, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(tmp_path_factory):
    rng = np.random.default_rng(3)
    alb = rng.uniform(0.2, 0.8, (4, synth.ALBEDO_BINS))
    th = rng.uniform(300.0, 600.0, (8, 8))
    sc = inverse.DiffScene(alb, th, width=48, spp=16, bounces=4,
                           out_dir=str(tmp_path_factory.mktemp("diff")))
    return sc, alb, th


def test_update_materials_equals_upload(small):
    sc, alb, th = small
    sc.set_params(alb * 0.9, th + 20.0)
    a = sc.render(seed=3)
    sc.ctx.upload(sc.flat)
    b = sc.render(seed=3)
    assert np.array_equal(a, b)
    sc.set_params(alb, th)


def test_autograd_function_backward(small):
    import torch
    sc, alb, th = small
    fn = inverse.render_fn()
    a = torch.tensor(alb, dtype=torch.float32, requires_grad=True)
    t = torch.tensor(th, dtype=torch.float32, requires_grad=True)
    w = torch.from_numpy(np.random.default_rng(1).standard_normal(sc.shape).astype(np.float32))
    img = fn.apply(a, t, sc, 5)
    assert img.shape == sc.shape
    (img * w).sum().backward()
    g_alb, g_th = sc.gradients(w.numpy(), seed=5 + 0x9E3779B9)
    # the gradients are sums of float atomics in arrival order: equal to
    # about 1e-4 of the largest entry between two runs of the same paths
    assert np.allclose(a.grad.numpy(), g_alb, rtol=1e-3, atol=1e-4 * np.abs(g_alb).max())
    assert np.allclose(t.grad.numpy(), g_th, rtol=1e-3, atol=1e-4 * np.abs(g_th).max())
    assert np.abs(g_th).max() > 0 and np.abs(g_alb).max() > 0


def test_inverse_loss_decreases():
    hist = inverse.run_inverse(iters=6, width=48, spp=8, target_spp=256, grid=8, n_spheres=4,
                               log=lambda *a: None)
    assert hist[-1][0] < hist[0][0]
