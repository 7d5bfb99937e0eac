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


MISS = np.uint32(0xFFFFFFFF)


def _mat(T):
    return np.asarray(T.M, np.float64).reshape(4, 4), np.asarray(T.M_inv, np.float64).reshape(4, 4)


def light_shadow_rays(sc, hits, seed=7):
    """Shadow rays from the hit points of a trace, built like
    sample::quaddirlight and sample::spherelight (cg.hpp:1625-1701): a light
    drawn uniformly, a point on a quad light (on a sphere light: a point of
    the sphere), the normalised direction to it, the distance bound (to the
    point, or to the sphere's centre as the reference uses) and the light's
    own object to skip.  Returns (rays, tmax, skip)."""
    rng = np.random.default_rng(seed)
    lights = [l for l in sc.lights if l.kind in ("quaddir", "sphere")]
    ok = hits["obj"] != MISS
    p = hits["p"][ok].astype(np.float32)
    n = p.shape[0]
    pick = rng.integers(0, len(lights), n)
    target = np.zeros((n, 3), np.float32)
    tmax = np.zeros(n, np.float32)
    skip = np.zeros(n, np.uint32)
    for k, l in enumerate(lights):
        sel = pick == k
        m = int(sel.sum())
        M, _ = _mat(l.T)
        pos = M[:3, 3]
        if l.kind == "quaddir":
            sx, sy = rng.uniform(-1, 1, (2, m))
            x = pos + sx[:, None] * M[:3, 0] + sy[:, None] * M[:3, 1]
            target[sel] = x
            tmax[sel] = np.linalg.norm(x - p[sel], axis=1)
        else:
            off = rng.normal(size=(m, 3))
            off /= np.linalg.norm(off, axis=1, keepdims=True)
            x = pos + off * float(l.size) * rng.uniform(0, 1, (m, 1))
            target[sel] = x
            tmax[sel] = np.linalg.norm(pos - p[sel], axis=1)
        skip[sel] = np.uint32(l.obj)
    d = (target - p).astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([p, d.astype(np.float32)], 1).astype(np.float32)
    return rays, tmax.astype(np.float32), skip


def overlap_origin_rays(sc, n, seed=8):
    """Rays in random directions from points that lie inside the bounds of
    at least two mesh objects at once: for these the reference's answer can
    depend on its object order (cg.hpp:1393, 1414), which the device
    resolves with its order checks and its linear-loop fallback.  Points are
    drawn in the intersections of the objects' world boxes and kept where
    both objects' local bounds contain them."""
    rng = np.random.default_rng(seed)
    objs = [(o, sc.meshes[o.mesh].bounds) for o in sc.objects if o.kind == "trimesh"]
    corners = np.array([[x, y, z, 1.0] for x in (0, 1) for y in (0, 1) for z in (0, 1)])
    wb = []
    for o, b in objs:
        M, _ = _mat(o.T)
        c = np.where(corners[:, :3] > 0, b[3:], b[:3])
        w = np.concatenate([c, np.ones((8, 1))], 1) @ M[:3].T
        wb.append((w.min(0), w.max(0)))

    def inside(o, b, x):
        _, Mi = _mat(o.T)
        l = np.concatenate([x, np.ones((x.shape[0], 1))], 1) @ Mi[:3].T
        return np.all((l >= b[:3]) & (l <= b[3:]), axis=1)

    pts = []
    for i in range(len(objs)):
        for j in range(i + 1, len(objs)):
            lo = np.maximum(wb[i][0], wb[j][0])
            hi = np.minimum(wb[i][1], wb[j][1])
            if np.any(lo >= hi):
                continue
            x = rng.uniform(lo, hi, size=(256, 3))
            ok = inside(*objs[i], x) & inside(*objs[j], x)
            pts.append(x[ok])
    p = np.concatenate(pts) if pts else np.zeros((0, 3))
    p = p[rng.permutation(p.shape[0])][:n]
    if p.shape[0] < n:
        p = p[rng.integers(0, max(p.shape[0], 1), n)] if p.shape[0] else p
    p = p.astype(np.float32)
    d = rng.normal(size=(p.shape[0], 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([p, d], 1).astype(np.float32)
