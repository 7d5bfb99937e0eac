"""Path-replay adjoint (lgpu_adjoint) against central finite differences.

The loss is linear in the image, Loss = <w, I> with a fixed seeded weight
image w, so dLoss/dI = w.  Lambertian albedo bins, thin-film thickness and
the thin-film IOR do not change any sampling decision, so a render with the
same seed at π ± h gives the same paths (common random numbers) and the
central difference matches the adjoint of those very paths up to the
difference's truncation and rounding: the tolerance is 2% relative, at the
step h = 1e-3 (relative for thickness), with the image accumulated in
double precision (LGPU_FLAG_FP64_FILM) so that the film's float rounding
does not swamp differences of that size.  The same differences are also
taken of the C restatement of the reference's estimator (oracle/, pinned bit
for bit to the reference) run on the device's random streams with its FP64
film: the reference's estimator with common random numbers.
The lobe exponent α moves sampled directions, so its finite difference and
the adjoint (which holds sampling fixed) agree only in expectation; they are
compared at high spp with a statistical tolerance."""
import numpy as np
import pytest

from lambda_b200 import _lib as L
from lambda_b200.renderer import Context
from lambda_b200.scene import FlatScene, load_nls

pytestmark = pytest.mark.gpu

SPP, B, P, SEED = 64, 8, 0.8, 17
REL_TOL = 0.02
H_REL = 1e-3


@pytest.fixture(scope="module")
def setup(mixed_nls):
    sc = load_nls(mixed_nls)
    flat = FlatScene(sc)
    ctx = Context()
    ctx.upload(flat)
    w_, h_ = ctx.size
    wimg = np.random.default_rng(5).standard_normal((h_, w_, 3)).astype(np.float32)
    return ctx, flat, wimg


def loss(ctx, flat, wimg, spp=SPP, seed=SEED):
    ctx.upload(flat)
    img = ctx.render(spp, B, P, seed=seed, flags=L.FLAG_FP64_FILM)
    return float(np.sum(img * wimg))


def oracle_loss(flat, wimg, spp=SPP, seed=SEED):
    """The loss of the restatement's FP64 image on the device's streams."""
    from oracle import restatement as R
    img = R.Oracle(flat).render(spp, B, P, rng=R.RNG_PCG, seed=seed, fp64=True)
    return float(np.sum(img * wimg))


def central_fd(ctx, flat, wimg, set_value, x0, h, spp=SPP, seed=SEED, on_oracle=False):
    f = (lambda: oracle_loss(flat, wimg, spp, seed)) if on_oracle else (lambda: loss(ctx, flat, wimg, spp, seed))
    set_value(x0 + h)
    lp = f()
    set_value(x0 - h)
    lm = f()
    set_value(x0)
    ctx.upload(flat)
    return (lp - lm) / (2 * h)


def mats_of(flat, kind):
    return [i for i, m in enumerate(flat.sc.materials) if m.kind == kind]


def test_adjoint_primal_image_is_the_render(setup):
    ctx, flat, wimg = setup
    gs, gm, img = ctx.adjoint(SPP, B, P, wimg, seed=SEED, image=True)
    ref = ctx.render(SPP, B, P, seed=SEED)
    assert np.array_equal(img, ref)
    assert np.all(np.isfinite(gs)) and np.all(np.isfinite(gm))


def test_adjoint_matches_fd_albedo_bins(setup):
    ctx, flat, wimg = setup
    gs, gm = ctx.adjoint(SPP, B, P, wimg, seed=SEED)
    checked = 0
    for mi in mats_of(flat, "lambertian"):
        s = flat.materials[mi].spectrum[0]
        # the bins with the largest gradients of this albedo
        for b in np.argsort(-np.abs(gs[s]))[:4]:
            def set_bin(v, s=s, b=b):
                flat.spectra[s, b] = v
            x0 = float(flat.spectra[s, b])
            fd = central_fd(ctx, flat, wimg, set_bin, x0, H_REL * max(abs(x0), 0.1))
            assert abs(gs[s, b] - fd) <= REL_TOL * abs(fd) + 1e-6 * np.abs(gs).max(), (mi, b, gs[s, b], fd)
            checked += 1
    assert checked >= 8


def test_adjoint_matches_fd_thin_film(setup):
    ctx, flat, wimg = setup
    gs, gm = ctx.adjoint(SPP, B, P, wimg, seed=SEED)
    for mi in mats_of(flat, "thinfilm"):
        m = flat.materials[mi]

        def set_d(v, m=m):
            m.d = v
        fd = central_fd(ctx, flat, wimg, set_d, float(m.d), H_REL * float(m.d))
        assert abs(gm[mi, 0] - fd) <= REL_TOL * abs(fd), ("thickness", gm[mi, 0], fd)
        # film IOR: every bin of its spectrum shifted together
        s = m.spectrum[0]
        base = flat.spectra[s].copy()

        def set_ior(v, s=s, base=base):
            flat.spectra[s] = base + np.float32(v)
        fd = central_fd(ctx, flat, wimg, set_ior, 0.0, 1e-3)
        g = float(np.sum(gs[s], dtype=np.float64))
        assert abs(g - fd) <= REL_TOL * abs(fd), ("film ior", g, fd)


def test_adjoint_matches_fd_of_the_reference_estimator(setup):
    """The device adjoint against central differences of the restatement of
    the reference's estimator (pinned bit for bit to the reference) on the
    device's random streams, FP64 film, h = 1e-3: albedo bins, thin-film
    thickness and film IOR.  Both follow the same paths; they differ only
    where a transcendental function's last bit sends a later bounce another
    way, so the differences agree within the same 2 %."""
    ctx, flat, wimg = setup
    gs, gm = ctx.adjoint(SPP, B, P, wimg, seed=SEED)
    checks = []
    for mi in mats_of(flat, "lambertian"):
        s = flat.materials[mi].spectrum[0]
        for b in np.argsort(-np.abs(gs[s]))[:2]:
            def set_bin(v, s=s, b=b):
                flat.spectra[s, b] = v
            x0 = float(flat.spectra[s, b])
            fd = central_fd(ctx, flat, wimg, set_bin, x0, H_REL * max(abs(x0), 0.1), on_oracle=True)
            checks.append(("albedo", mi, b, float(gs[s, b]), fd))
    for mi in mats_of(flat, "thinfilm"):
        m = flat.materials[mi]

        def set_d(v, m=m):
            m.d = v
        fd = central_fd(ctx, flat, wimg, set_d, float(m.d), H_REL * float(m.d), on_oracle=True)
        checks.append(("thickness", mi, 0, float(gm[mi, 0]), fd))
        s = m.spectrum[0]
        base = flat.spectra[s].copy()

        def set_ior(v, s=s, base=base):
            flat.spectra[s] = base + np.float32(v)
        fd = central_fd(ctx, flat, wimg, set_ior, 0.0, H_REL, on_oracle=True)
        checks.append(("film ior", mi, 0, float(np.sum(gs[s], dtype=np.float64)), fd))
    print(checks)
    scale = max(abs(c[4]) for c in checks)
    for name, mi, b, g, fd in checks:
        assert abs(g - fd) <= REL_TOL * abs(fd) + 1e-6 * scale, (name, mi, b, g, fd)
    assert len(checks) >= 6


def test_adjoint_blinn_alpha_in_expectation(scene_dir):
    """Blinn lobe exponent α on a glossy floor lit and viewed from above
    (every half vector faces up, so pow(h·n, α) is defined for the
    non-integer α of a finite difference, cg.hpp:1810, 1822): the adjoint
    and central differences, each averaged over independent seeds, agree
    within 4 standard errors."""
    import json
    import os
    d = os.path.join(str(scene_dir), "glossy_floor")
    os.makedirs(d, exist_ok=True)
    scene = {"camera": {"pos": [0.0, -3.0, 2.5], "look_at": [0.0, 0.0, 0.0], "up": [0, 0, 1], "fov": 40,
                        "ar": 1.0, "width": 48},
             "materials": [{"name": "gloss", "type": "blinn", "Kd": {"val": 0.2}, "Ks": {"val": 0.6},
                            "glossiness": 24}],
             "objects": [{"name": "floor", "type": "plane", "transform": {"scale": [4, 4, 1]},
                          "material": "gloss"}],
             "lights": [{"name": "panel", "type": "quaddir", "specular": 2, "radiance": {"val": 4.0},
                         "transform": {"scale": [0.8, 0.8, 1], "rotate": {"axis": [1, 0, 0], "degrees": 180},
                                       "translate": [0.0, 1.5, 2.5]}}]}
    nls = os.path.join(d, "scene.nls")
    with open(nls, "w") as f:
        json.dump(scene, f)
    flat = FlatScene(load_nls(nls))
    ctx = Context()
    ctx.upload(flat)
    w_, h_ = ctx.size
    wimg = np.random.default_rng(9).standard_normal((h_, w_, 3)).astype(np.float32)
    mi = mats_of(flat, "blinn")[0]
    m = flat.materials[mi]
    a0 = float(m.alpha)

    def set_a(v):
        m.alpha = v
    spp, n_seeds = 256, 8
    adj = np.array([ctx.adjoint(spp, B, P, wimg, seed=3000 + k)[1][mi, 1] for k in range(n_seeds)], np.float64)
    fd = np.array([central_fd(ctx, flat, wimg, set_a, a0, 0.02 * a0, spp=spp, seed=4000 + k)
                   for k in range(n_seeds)])
    se = np.sqrt(adj.var(ddof=1) / n_seeds + fd.var(ddof=1) / n_seeds)
    print("blinn alpha", a0, adj.mean(), fd.mean(), se)
    assert np.all(np.isfinite(adj)) and np.all(np.isfinite(fd))
    assert abs(adj.mean()) > 4 * se  # the gradient is resolved, not noise
    assert abs(adj.mean() - fd.mean()) <= 4 * se, (adj.mean(), fd.mean(), se)


def test_adjoint_alpha_in_expectation(setup):
    """α: the adjoint holds sampling fixed, the finite difference lets the
    sampled directions move with α, so they agree in expectation only.
    Each is averaged over independent seeds; their difference must be within
    4 standard errors."""
    ctx, flat, wimg = setup
    spp, n_seeds = 512, 8
    # (Blinn lobes are left out: the reference's pow(h.n, α) of a
    # back-facing half vector is NaN for the non-even α of a finite
    # difference, cg.hpp:1810, 1822)
    for mi in mats_of(flat, "thinfilm"):
        m = flat.materials[mi]
        a0 = float(m.alpha)

        def set_a(v, m=m):
            m.alpha = v
        adj = np.array([ctx.adjoint(spp, B, P, wimg, seed=1000 + k)[1][mi, 1] for k in range(n_seeds)],
                       np.float64)
        fd = np.array([central_fd(ctx, flat, wimg, set_a, a0, 0.02 * a0, spp=spp, seed=2000 + k)
                       for k in range(n_seeds)])
        se = np.sqrt(adj.var(ddof=1) / n_seeds + fd.var(ddof=1) / n_seeds)
        print("alpha", mi, a0, adj.mean(), fd.mean(), se)
        assert abs(adj.mean() - fd.mean()) <= 4 * se + 1e-9, (mi, adj.mean(), fd.mean(), se)
