"""Inverse rendering on the device: a torch.autograd.Function whose forward
is the spectral path tracer (lgpu_render) and whose backward is its
path-replay adjoint (lgpu_adjoint), and a harness that recovers the
thin-film thickness map and the sphere albedos of lambda_b200.synth's
diff_scene from a target image.

    python -m lambda_b200.inverse --iters 20 --width 128 --spp 8

Parameters: albedo (n_spheres, 32) samples on 400-720 nm, mapped to the
renderer's 80 bins by the reference's box average (a linear map, the same
one the .nls loader applies to a 32-sample CSV), and thickness (G, G) nm.
"""
import argparse
import os
import tempfile
import time

import numpy as np

from . import synth
from .renderer import Context
from .scene import FlatScene, coef_from_samples, load_nls


def albedo_map(cfg, n=synth.ALBEDO_BINS):
    """(n_bins, n) matrix A with coefficientλ(samples v) = A v for samples
    at synth.albedo_wavelengths(n) (cg.hpp:252-272 is linear in v)."""
    lam = synth.albedo_wavelengths(n)
    A = np.zeros((cfg.n_bins, n), np.float64)
    for i in range(n):
        e = np.zeros(n)
        e[i] = 1.0
        A[:, i] = coef_from_samples(lam, e, cfg)
    return A


class DiffScene:
    """diff_scene on one device: the uploaded scene, where its parameters
    live in the flat tables, and the render settings."""

    def __init__(self, albedo, thickness, width=512, spp=32, bounces=4, sample_p=0.8, device=0,
                 out_dir=None):
        self.G = int(np.asarray(thickness).shape[0])
        out_dir = out_dir or os.path.join(tempfile.gettempdir(), "lgpu_diff_%d_%d" % (self.G, width))
        nls = synth.diff_scene(out_dir, albedo, thickness, width=width)
        self.sc = load_nls(nls)
        self.flat = FlatScene(self.sc)
        self.ctx = Context(device)
        self.ctx.upload(self.flat)
        mats = self.sc.materials
        self.film = np.array([i for i, m in enumerate(mats) if m.kind == "thinfilm"])
        self.alb = np.array([i for i, m in enumerate(mats) if m.kind == "lambertian"])
        self.alb_rows = np.array([self.flat.materials[i].spectrum[0] for i in self.alb])
        self.A = albedo_map(self.sc.cfg)
        self.spp, self.bounces, self.p = spp, bounces, sample_p
        self.shape = (self.ctx.size[1], self.ctx.size[0], 3)

    def set_params(self, albedo, thickness):
        """Writes the parameters into the flat tables and the device."""
        spec = np.asarray(albedo, np.float64) @ self.A.T
        self.flat.spectra[self.alb_rows] = spec.astype(np.float32)
        th = np.asarray(thickness, np.float64).reshape(-1)
        for k, mi in enumerate(self.film):
            self.flat.materials[int(mi)].d = float(th[k])
        self.ctx.update_materials(self.flat)

    def render(self, seed, spp=None):
        return self.ctx.render(spp or self.spp, self.bounces, self.p, seed=seed)

    def gradients(self, dloss_dimage, seed, spp=None):
        """(dLoss/dalbedo (n, 32), dLoss/dthickness (G, G))."""
        gs, gm = self.ctx.adjoint(spp or self.spp, self.bounces, self.p, dloss_dimage, seed=seed)
        g_alb = gs[self.alb_rows].astype(np.float64) @ self.A
        g_th = gm[self.film, 0].astype(np.float64).reshape(self.G, self.G)
        return g_alb, g_th


def _torch_function():
    import torch

    class RenderFunction(torch.autograd.Function):
        """image = render(albedo, thickness); backward by path replay with
        a seed of its own (the image and the gradient use independent paths,
        so the gradient of an L2 loss is unbiased)."""

        @staticmethod
        def forward(ctx, albedo, thickness, scene, seed):
            scene.set_params(albedo.detach().cpu().numpy(), thickness.detach().cpu().numpy())
            img = scene.render(seed)
            ctx.scene, ctx.seed = scene, seed
            ctx.dev = albedo.device
            return torch.from_numpy(img).to(albedo.device)

        @staticmethod
        def backward(ctx, grad_img):
            g = grad_img.detach().float().cpu().numpy()
            g_alb, g_th = ctx.scene.gradients(g, seed=ctx.seed + 0x9E3779B9)
            return (torch.from_numpy(g_alb).float().to(ctx.dev), torch.from_numpy(g_th).float().to(ctx.dev),
                    None, None)

    return RenderFunction


RenderFunction = None


def render_fn():
    global RenderFunction
    if RenderFunction is None:
        RenderFunction = _torch_function()
    return RenderFunction


def run_inverse(iters=20, width=128, spp=8, target_spp=1024, grid=64, n_spheres=64, lr_th=15.0, lr_alb=0.03,
                seed=0, log=print):
    """Recovers hidden thickness / albedo from a target rendered at
    target_spp; returns the loss and parameter-error history."""
    import torch
    rng = np.random.default_rng(seed)
    th_true = rng.uniform(200.0, 800.0, (grid, grid))
    alb_true = np.clip(0.15 + 0.7 * rng.uniform(size=(n_spheres, 1)) +
                       0.1 * np.sin(np.linspace(0, 3, synth.ALBEDO_BINS)[None, :] * rng.uniform(1, 3, (n_spheres, 1))),
                       0.05, 0.95)
    scene = DiffScene(np.full((n_spheres, synth.ALBEDO_BINS), 0.5), np.full((grid, grid), 400.0), width=width,
                      spp=spp)
    scene.set_params(alb_true, th_true)
    target = torch.from_numpy(scene.render(seed=12345, spp=target_spp))
    alb = torch.full((n_spheres, synth.ALBEDO_BINS), 0.5, dtype=torch.float32, requires_grad=True)
    th = torch.full((grid, grid), 400.0, dtype=torch.float32, requires_grad=True)
    opt = torch.optim.Adam([{"params": [alb], "lr": lr_alb}, {"params": [th], "lr": lr_th}])
    fn = render_fn()
    hist = []
    for it in range(iters):
        t0 = time.perf_counter()
        opt.zero_grad()
        img = fn.apply(alb, th, scene, 1000 + it)
        loss = torch.mean((img - target) ** 2)
        loss.backward()
        opt.step()
        with torch.no_grad():
            alb.clamp_(0.0, 1.0)
            th.clamp_(100.0, 900.0)
        err_th = float(np.sqrt(np.mean((th.detach().numpy() - th_true) ** 2)))
        err_alb = float(np.sqrt(np.mean((alb.detach().numpy() - alb_true) ** 2)))
        hist.append((float(loss.detach()), err_th, err_alb))
        log("iter %3d  loss %.6e  thickness rmse %.1f nm  albedo rmse %.4f  (%.2f s)" %
            (it, hist[-1][0], err_th, err_alb, time.perf_counter() - t0))
    return hist


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--width", type=int, default=128)
    ap.add_argument("--spp", type=int, default=8)
    ap.add_argument("--target-spp", type=int, default=1024)
    ap.add_argument("--grid", type=int, default=64)
    args = ap.parse_args()
    run_inverse(args.iters, args.width, args.spp, args.target_spp, args.grid)


if __name__ == "__main__":
    main()
