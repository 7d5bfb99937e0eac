"""Deterministic ray sets for closest-hit parity tests."""
import numpy as np


def camera_rays(sc, n_per_axis=64, seed=0):
    """Rays through a jittered grid of the camera's image plane, built like
    sample::camera (cg.hpp:1534-1542) with a pinhole."""
    rng = np.random.default_rng(seed)
    cam = sc.cam
    x, y, z = (np.array(v, np.float32) for v in cam.base)
    pos = np.array(cam.pos, np.float32)
    u = (np.arange(n_per_axis) + rng.random(n_per_axis)) / n_per_axis * cam.width
    v = (np.arange(n_per_axis) + rng.random(n_per_axis)) / n_per_axis * cam.height
    U, Vv = np.meshgrid(u, v)
    U, Vv = U.ravel().astype(np.float32), Vv.ravel().astype(np.float32)
    a = (-0.5 * cam.w + cam.delta * U)[:, None]
    b = (-0.5 * cam.h + cam.delta * Vv)[:, None]
    wij = pos + x * a + y * b - cam.D * z
    d = wij - pos
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([np.repeat(pos[None], d.shape[0], 0), d], 1).astype(np.float32)


def bounce_rays(hits, seed=1):
    """Rays from the hit points of a previous trace in random directions
    (both hemispheres), like extension and shadow rays of a path."""
    rng = np.random.default_rng(seed)
    ok = hits["obj"] != np.uint32(0xFFFFFFFF)
    p = hits["p"][ok]
    d = rng.normal(size=(p.shape[0], 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([p, d], 1).astype(np.float32)


def random_rays(lo, hi, n, seed=2):
    rng = np.random.default_rng(seed)
    p = rng.uniform(lo, hi, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    # some axis-aligned directions exercise the inv_u = FLT_MAX branch
    k = n // 16
    d[:k] = 0.0
    d[np.arange(k), rng.integers(0, 3, k)] = rng.choice([-1.0, 1.0], k)
    return np.concatenate([p, d], 1).astype(np.float32)
