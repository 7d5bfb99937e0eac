"""Seeded synthetic scenes for the benchmark configurations.

Each generator writes a self-contained scene directory — scene.nls with
absolute paths, triangle OBJ files with per-vertex normals, spectra as
'λ,value' CSV files — that both the reference loader (load::loadNLS,
cg.hpp:2455) and lambda_b200.scene.load_nls read.  The reference ships no
benchmark scenes of these shapes; these stand in for them:

  box_room   unit cube of 5 interior walls (10 triangles: white 0.75, left
             0.6 above 600 nm / 0.05 below, right 0.6 in 500-560 nm / 0.05
             elsewhere), two axis-aligned blocks (12 triangles each,
             0.3x0.3x0.6 and 0.3x0.3x0.3, 0.75), a 0.25x0.25 ceiling quad
             light with 6500 K blackbody emission.
  instanced  N instances of one seeded displaced icosphere (subdivision s:
             20*4^s triangles, Perlin displacement amplitude 0.05) on a
             2-triangle ground plane under 2 quad lights; materials drawn
             uniformly from Lambertian (smooth random spectra 0.05-0.9),
             Blinn (exponent log-uniform 8-2048) and thin film (thickness
             U[200,800] nm, IOR U[1.33,1.6]).
"""
import json
import os

import numpy as np

from .scene import write_obj

H_PLANCK = 6.62607015e-34
C_LIGHT = 2.99792458e8
K_BOLTZ = 1.380649e-23


def planck(lam_nm, T):
    lam = np.asarray(lam_nm, np.float64) * 1e-9
    return 2 * H_PLANCK * C_LIGHT ** 2 / lam ** 5 / np.expm1(H_PLANCK * C_LIGHT / (lam * K_BOLTZ * T))


def write_csv(path, lam, val):
    with open(path, "w") as f:
        for l, v in zip(lam, val):
            f.write("%.1f,%.6f\n" % (l, v))


def blackbody_csv(path, T, peak=1.0):
    """Planck radiance at temperature T on 300-830 nm, scaled so that its
    value at 560 nm is `peak`."""
    lam = np.arange(300.0, 835.0, 5.0)
    b = planck(lam, T)
    b = b / planck([560.0], T)[0] * peak
    write_csv(path, lam, b)


def step_csv(path, lo, hi, inside, outside):
    """inside on [lo, hi] nm, outside elsewhere, as a step sampled finely."""
    lam, val = [], []
    for l in np.arange(300.0, 835.0, 1.0):
        lam.append(l)
        val.append(inside if lo <= l <= hi else outside)
    write_csv(path, lam, val)


def smooth_random_csv(path, rng, lo=0.05, hi=0.9):
    """A smooth random reflectance on 380-780 nm at 5 nm (81 samples):
    a few random Gaussian bumps, rescaled into [lo, hi]."""
    lam = np.arange(380.0, 785.0, 5.0)
    v = np.zeros_like(lam)
    for _ in range(3):
        c = rng.uniform(380, 780)
        w = rng.uniform(30, 120)
        v += rng.uniform(0.2, 1.0) * np.exp(-0.5 * ((lam - c) / w) ** 2)
    v = (v - v.min()) / max(v.max() - v.min(), 1e-6)
    a, b = sorted(rng.uniform(lo, hi, size=2))
    if b - a < 0.1:
        b = min(hi, a + 0.1)
    v = a + (b - a) * v
    write_csv(path, lam, v)
    return v


def _quad(p0, p1, p2, p3):
    """Two triangles of the quad p0 p1 p2 p3 (counter-clockwise seen from the
    side its normal points to)."""
    return [p0, p1, p2, p3], [(0, 1, 2), (0, 2, 3)]


def _write_flat_mesh(path, quads):
    """OBJ of planar quads with one flat normal per quad: normal = (p1-p0) x
    (p2-p0), the geometric normal the reference loader computes.

    A mesh's bounds include fast_obj's dummy vertex at the origin
    (cg.hpp:2215-2229), and the reference never hits a mesh whose bounds
    are flat (its slab test needs t_min < t_max, cg.hpp:1268-1286): a single
    quad through the origin's plane is therefore written one unit off that
    plane and moved back by its object transform."""
    V, N, F = [], [], []
    for q in quads:
        base = len(V)
        p = [np.asarray(x, np.float64) for x in q]
        n = np.cross(p[1] - p[0], p[2] - p[0])
        n /= np.linalg.norm(n)
        V.extend(p)
        N.append(n)
        ni = len(N)
        F.append((base + 1, base + 2, base + 3, ni, ni, ni))
        F.append((base + 1, base + 3, base + 4, ni, ni, ni))
    write_obj(path, V, N, F)


def _box_quads(lo, hi, inward=False):
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    quads = [
        [(x0, y0, z0), (x0, y1, z0), (x1, y1, z0), (x1, y0, z0)],  # bottom (-z)
        [(x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)],  # top (+z)
        [(x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1)],  # front (-y)
        [(x0, y1, z0), (x0, y1, z1), (x1, y1, z1), (x1, y1, z0)],  # back (+y)
        [(x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0)],  # left (-x)
        [(x1, y0, z0), (x1, y1, z0), (x1, y1, z1), (x1, y0, z1)],  # right (+x)
    ]
    if inward:
        quads = [q[::-1] for q in quads]
    return quads


def _mat_spec(path):
    return {"val": path}


def box_room(out_dir, width=256, light_peak=6.0):
    """Writes the box-room scene; returns the .nls path."""
    os.makedirs(out_dir, exist_ok=True)
    d = os.path.abspath(out_dir)
    walls = _box_quads((0, 0, 0), (1, 1, 1), inward=True)
    # inward walls: bottom, top, back, left, right (the -y side is open)
    white = [walls[0], walls[1], walls[3]]
    _write_flat_mesh(os.path.join(d, "walls_white.obj"), white)
    # the left wall lies in the plane x = 0 of the dummy vertex: written at
    # x = 1 and moved back by the object transform
    _write_flat_mesh(os.path.join(d, "wall_left.obj"), [[(x + 1, y, z) for (x, y, z) in walls[4]]])
    _write_flat_mesh(os.path.join(d, "wall_right.obj"), [walls[5]])
    _write_flat_mesh(os.path.join(d, "block_tall.obj"),
                     _box_quads((0.2, 0.45, 0.0), (0.5, 0.75, 0.6)))
    _write_flat_mesh(os.path.join(d, "block_short.obj"),
                     _box_quads((0.58, 0.2, 0.0), (0.88, 0.5, 0.3)))
    step_csv(os.path.join(d, "left.csv"), 600.0, 10000.0, 0.6, 0.05)
    step_csv(os.path.join(d, "right.csv"), 500.0, 560.0, 0.6, 0.05)
    blackbody_csv(os.path.join(d, "bb6500.csv"), 6500.0, light_peak)
    scene = {
        "camera": {"pos": [0.5, -1.4, 0.5], "look_at": [0.5, 0.5, 0.5], "up": [0, 0, 1],
                   "fov": 40, "ar": 1.0, "width": width},
        "materials": [
            {"name": "white", "type": "lambertian", "albedo": {"val": 0.75}},
            {"name": "left", "type": "lambertian", "albedo": _mat_spec(os.path.join(d, "left.csv"))},
            {"name": "right", "type": "lambertian",
             "albedo": _mat_spec(os.path.join(d, "right.csv"))},
        ],
        "objects": [
            {"name": "walls", "type": "trimesh", "transform": {},
             "material": "white", "source": os.path.join(d, "walls_white.obj")},
            {"name": "left", "type": "trimesh", "transform": {"translate": [-1, 0, 0]},
             "material": "left", "source": os.path.join(d, "wall_left.obj")},
            {"name": "right", "type": "trimesh", "transform": {},
             "material": "right", "source": os.path.join(d, "wall_right.obj")},
            {"name": "tall", "type": "trimesh", "transform": {},
             "material": "white", "source": os.path.join(d, "block_tall.obj")},
            {"name": "short", "type": "trimesh", "transform": {},
             "material": "white", "source": os.path.join(d, "block_short.obj")},
        ],
        "lights": [
            {"name": "ceiling", "type": "quaddir", "specular": 2,
             "transform": {"scale": [0.125, 0.125, 1], "rotate": {"axis": [1, 0, 0], "degrees": 180},
                           "translate": [0.5, 0.5, 0.998]},
             "radiance": {"val": os.path.join(d, "bb6500.csv")}},
        ],
    }
    path = os.path.join(d, "scene.nls")
    with open(path, "w") as f:
        json.dump(scene, f, indent=1)
    return path


# ---- displaced icosphere ---------------------------------------------------------

def icosphere(subdiv):
    """Unit icosphere: 20*4^subdiv triangles, outward winding."""
    t = (1.0 + 5 ** 0.5) / 2.0
    V = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
         (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
         (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    V = np.array(V, np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array(F, np.int64)
    for _ in range(subdiv):
        nv = V.shape[0]
        e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        key = np.minimum(e[:, 0], e[:, 1]) * (nv + 1) + np.maximum(e[:, 0], e[:, 1])
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq // (nv + 1)
        b = uniq % (nv + 1)
        mid = V[a] + V[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        mids = nv + inv.reshape(3, -1).T  # (n_faces, 3): m01, m12, m20
        V = np.concatenate([V, mid])
        f0, f1, f2 = F[:, 0], F[:, 1], F[:, 2]
        m01, m12, m20 = mids[:, 0], mids[:, 1], mids[:, 2]
        F = np.concatenate([np.stack([f0, m01, m20], 1), np.stack([f1, m12, m01], 1),
                            np.stack([f2, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return V, F


def perlin3(p, perm):
    """Improved Perlin noise (Perlin 2002) at points p (n, 3)."""
    def fade(t):
        return t * t * t * (t * (t * 6 - 15) + 10)

    def grad(h, x, y, z):
        h = h & 15
        u = np.where(h < 8, x, y)
        v = np.where(h < 4, y, np.where((h == 12) | (h == 14), x, z))
        return np.where(h & 1, -u, u) + np.where(h & 2, -v, v)

    P = np.floor(p).astype(np.int64)
    f = p - P
    X, Y, Z = (P[:, 0] & 255), (P[:, 1] & 255), (P[:, 2] & 255)
    x, y, z = f[:, 0], f[:, 1], f[:, 2]
    u, v, w = fade(x), fade(y), fade(z)
    pp = np.concatenate([perm, perm])
    A = pp[X] + Y
    AA, AB = pp[A] + Z, pp[A + 1] + Z
    B = pp[X + 1] + Y
    BA, BB = pp[B] + Z, pp[B + 1] + Z

    def lerp(t, a, b):
        return a + t * (b - a)

    return lerp(w, lerp(v, lerp(u, grad(pp[AA], x, y, z), grad(pp[BA], x - 1, y, z)),
                        lerp(u, grad(pp[AB], x, y - 1, z), grad(pp[BB], x - 1, y - 1, z))),
                lerp(v, lerp(u, grad(pp[AA + 1], x, y, z - 1), grad(pp[BA + 1], x - 1, y, z - 1)),
                     lerp(u, grad(pp[AB + 1], x, y - 1, z - 1), grad(pp[BB + 1], x - 1, y - 1, z - 1))))


def displaced_icosphere(subdiv, seed, amp=0.05, freq=3.0):
    """Icosphere displaced along its normal by amp * Perlin(freq * p); vertex
    normals are area-weighted face normals of the displaced surface."""
    V, F = icosphere(subdiv)
    return _displace(V, F, seed, amp, freq)


def displaced_uv_sphere(seed, n_lon=256, n_lat=129, amp=0.05, freq=3.0):
    """UV sphere of n_lon * (n_lat - 2) * 2 + 2 * n_lon triangles (65,536 by
    default) displaced as displaced_icosphere."""
    V, _, F = uv_sphere(n_lon, n_lat)
    return _displace(V, F, seed, amp, freq)


def _displace(V, F, seed, amp, freq):
    rng = np.random.default_rng(seed)
    perm = rng.permutation(256)
    n = perlin3(V * freq + rng.uniform(0, 100, size=3), perm)
    V = V * (1.0 + amp * n)[:, None]
    e0 = V[F[:, 1]] - V[F[:, 0]]
    e2 = V[F[:, 2]] - V[F[:, 0]]
    fn = np.cross(e0, e2)
    N = np.zeros_like(V)
    for k in range(3):
        np.add.at(N, F[:, k], fn)
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    return V, N, F


def write_indexed_obj(path, V, N, F):
    """OBJ with shared vertices: face corner k uses position and normal k."""
    Fo = np.concatenate([F + 1, F + 1], axis=1)
    write_obj(path, V, N, Fo)


def mixed(out_dir, width=96, ar=1.25, lights=("sphere", "quaddir", "point"), seed=7,
          subdiv=3, dof=None, focal=None):
    """A small scene with every object kind (sphere, plane, instanced
    trimesh), every shaded material (Lambertian, Blinn reflective/diffuse,
    Blinn refractive with a dispersive IOR, thin film) and the requested
    light kinds (sphere, quaddir, point, direction, ambient).  With dof, a
    thin-lens camera of that aperture focused at distance `focal` (the
    camera's "dof" and "f", cg.hpp:2050-2051, sampled at cg.hpp:1539).
    Returns the .nls path."""
    os.makedirs(out_dir, exist_ok=True)
    d = os.path.abspath(out_dir)
    rng = np.random.default_rng(seed)
    mesh = os.path.join(d, f"ico_s{subdiv}.obj")
    V, N, F = displaced_icosphere(subdiv, seed, amp=0.08)
    write_indexed_obj(mesh, V, N, F)
    smooth_random_csv(os.path.join(d, "albedo.csv"), rng, 0.1, 0.8)
    blackbody_csv(os.path.join(d, "bb.csv"), 5000.0, 4.0)
    lam = np.arange(330.0, 800.0, 10.0)
    write_csv(os.path.join(d, "glass_ior.csv"), lam, 1.5 + 4000.0 / lam ** 2)
    write_csv(os.path.join(d, "film_ior.csv"), lam, 1.35 + 2000.0 / lam ** 2)
    mats = [
        {"name": "floor", "type": "lambertian", "albedo": {"val": [0.6, 0.55, 0.5]}},
        {"name": "wall", "type": "lambertian", "albedo": {"val": os.path.join(d, "albedo.csv")}},
        {"name": "gloss", "type": "blinn", "Kd": {"val": [0.7, 0.3, 0.1]}, "Ks": {"val": 0.3},
         "glossiness": 64},
        {"name": "mirror", "type": "blinn", "Ks": {"val": 0.9}, "glossiness": 512},
        {"name": "glass", "type": "blinn", "Kt": {"val": 0.9}, "Kd": {"val": 0.02},
         "glossiness": 2048, "ior": {"val": os.path.join(d, "glass_ior.csv")}},
        {"name": "film", "type": "thinfilm", "glossiness": 256, "thickness": 480,
         "film_ior": {"val": os.path.join(d, "film_ior.csv")}, "base_ior": {"val": 1.6}},
    ]
    objs = [
        {"name": "floor", "type": "plane", "transform": {"scale": [8, 8, 1]}, "material": "floor"},
        {"name": "back", "type": "plane", "material": "wall",
         "transform": {"scale": [8, 4, 1], "rotate": {"axis": [1, 0, 0], "degrees": 90},
                       "translate": [0, 3, 4]}},
        {"name": "ball", "type": "sphere", "material": "gloss",
         "transform": {"scale": [0.8, 0.8, 0.8], "translate": [-1.6, 0.2, 0.8]}},
        {"name": "chrome", "type": "sphere", "material": "mirror",
         "transform": {"scale": [0.6, 0.6, 0.6], "translate": [1.7, 1.0, 0.6]}},
        {"name": "rock1", "type": "trimesh", "material": "glass", "source": mesh,
         "transform": {"scale": [0.9, 0.9, 0.9], "rotate": {"axis": [0, 1, 1], "degrees": 30},
                       "translate": [0.1, -0.4, 0.9]}},
        {"name": "rock2", "type": "trimesh", "material": "film", "source": mesh,
         "transform": {"scale": [0.7, 0.5, 0.7], "rotate": {"axis": [1, 0, 0], "degrees": -20},
                       "translate": [1.2, -1.3, 0.5]}},
    ]
    ls = []
    for kind in lights:
        if kind == "sphere":
            ls.append({"name": "sun", "type": "sphere", "radiance": {"val": 6.0},
                       "transform": {"scale": [0.5, 0.5, 0.5], "translate": [-2.5, -1.5, 4.0]}})
        elif kind == "quaddir":
            ls.append({"name": "panel", "type": "quaddir", "specular": 2,
                       "radiance": {"val": os.path.join(d, "bb.csv")},
                       "transform": {"scale": [0.8, 0.6, 1],
                                     "rotate": {"axis": [1, 0, 0], "degrees": 160},
                                     "translate": [1.5, -0.5, 3.5]}})
        elif kind == "point":
            ls.append({"name": "bulb", "type": "point", "radiant_intensity": {"val": 3.0},
                       "pos": [0.5, -2.5, 2.5]})
        elif kind == "direction":
            ls.append({"name": "sky", "type": "direction", "radiant_intensity": {"val": 0.8},
                       "dir": [0.3, 0.4, -0.866]})
        elif kind == "ambient":
            ls.append({"name": "amb", "type": "ambient", "radiance": {"val": 0.15}})
    scene = {"camera": {"pos": [0.0, -6.0, 2.2], "look_at": [0.0, 0.0, 0.8], "up": [0, 0, 1],
                        "fov": 45, "ar": ar, "width": width},
             "materials": mats, "objects": objs, "lights": ls}
    if dof is not None:
        scene["camera"]["dof"] = float(dof)
        scene["camera"]["f"] = float(focal if focal is not None else 6.0)
    path = os.path.join(d, "scene.nls")
    with open(path, "w") as f:
        json.dump(scene, f, indent=1)
    return path


def instanced(out_dir, n_instances=64, subdiv=7, seed=1234, width=1920, ar=16 / 9, mesh="icosphere"):
    """Writes the instanced scene; returns the .nls path.  mesh: "icosphere"
    (subdivision subdiv) or "uv64k" (the 65,536-triangle displaced UV
    sphere)."""
    os.makedirs(out_dir, exist_ok=True)
    d = os.path.abspath(out_dir)
    rng = np.random.default_rng(seed)
    if mesh == "uv64k":
        mesh_path = os.path.join(d, f"uvsphere64k_seed{seed}.obj")
        if not os.path.exists(mesh_path):
            V, N, F = displaced_uv_sphere(seed)
            write_indexed_obj(mesh_path, V, N, F)
    else:
        mesh_path = os.path.join(d, f"icosphere_s{subdiv}_seed{seed}.obj")
        if not os.path.exists(mesh_path):
            V, N, F = displaced_icosphere(subdiv, seed)
            write_indexed_obj(mesh_path, V, N, F)
    # written at z = 1, moved to z = 0 by the object transform (flat bounds
    # through the dummy vertex are never hit, see _write_flat_mesh)
    _write_flat_mesh(os.path.join(d, "ground.obj"),
                     [[(-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)]])
    blackbody_csv(os.path.join(d, "bb6500.csv"), 6500.0, 3.0)
    blackbody_csv(os.path.join(d, "bb4000.csv"), 4000.0, 2.0)
    materials = [{"name": "ground", "type": "lambertian", "albedo": {"val": 0.5}}]
    objects = [{"name": "ground", "type": "trimesh", "material": "ground",
                "transform": {"scale": [12, 12, 1], "translate": [0, 0, -1]},
                "source": os.path.join(d, "ground.obj")}]
    side = int(np.ceil(np.sqrt(n_instances)))
    spacing = 1.1
    for i in range(n_instances):
        kind = ["lambertian", "blinn", "thinfilm"][int(rng.integers(0, 3))]
        name = f"m{i}"
        if kind == "lambertian":
            p = os.path.join(d, f"albedo_{i}.csv")
            smooth_random_csv(p, rng)
            materials.append({"name": name, "type": "lambertian", "albedo": {"val": p}})
        elif kind == "blinn":
            p = os.path.join(d, f"kd_{i}.csv")
            smooth_random_csv(p, rng, 0.05, 0.6)
            # an even integer exponent keeps powf defined for back-facing
            # half vectors (cg.hpp:1810, 1822)
            alpha = 2 * int(round(np.exp(rng.uniform(np.log(8), np.log(2048))) / 2))
            materials.append({"name": name, "type": "blinn", "Kd": {"val": p},
                              "Ks": {"val": float(rng.uniform(0.2, 0.5))}, "glossiness": alpha})
        else:
            alpha = 2 * int(round(np.exp(rng.uniform(np.log(8), np.log(2048))) / 2))
            materials.append({"name": name, "type": "thinfilm",
                              "film_ior": {"val": float(rng.uniform(1.33, 1.6))},
                              "base_ior": {"val": 1.5}, "glossiness": alpha,
                              "thickness": float(rng.uniform(200, 800))})
        gx, gy = i % side, i // side
        s = 0.45
        objects.append({"name": f"inst{i}", "type": "trimesh", "material": name,
                        "source": mesh_path,
                        "transform": {"scale": [s, s, s],
                                      "rotate": {"axis": [0, 0, 1],
                                                 "degrees": float(rng.uniform(0, 360))},
                                      "translate": [(gx - (side - 1) / 2) * spacing,
                                                    (gy - (side - 1) / 2) * spacing, s]}})
    lights = [
        {"name": "key", "type": "quaddir", "specular": 2,
         "transform": {"scale": [1.5, 1.5, 1], "rotate": {"axis": [1, 0, 0], "degrees": 180},
                       "translate": [-2.0, -1.0, 6.0]},
         "radiance": {"val": os.path.join(d, "bb6500.csv")}},
        {"name": "fill", "type": "quaddir", "specular": 2,
         "transform": {"scale": [1.0, 1.0, 1], "rotate": {"axis": [1, 0, 0], "degrees": 180},
                       "translate": [3.0, 2.0, 5.0]},
         "radiance": {"val": os.path.join(d, "bb4000.csv")}},
    ]
    extent = side * spacing
    scene = {
        "camera": {"pos": [0.0, -0.95 * extent, 0.75 * extent], "look_at": [0, 0, 0.2],
                   "up": [0, 0, 1], "fov": 50, "ar": ar, "width": width},
        "materials": materials, "objects": objects, "lights": lights,
    }
    path = os.path.join(d, "scene.nls")
    with open(path, "w") as f:
        json.dump(scene, f, indent=1)
    return path


def batch_job(out_dir, n_instances, subdiv, mesh_dir, seed, width):
    """A batched-render job scene: the box room with n_instances copies of a
    displaced icosphere (subdivision subdiv, shared by every job through
    mesh_dir) standing on its floor, materials drawn as in instanced();
    returns the .nls path."""
    base = box_room(out_dir, width=width)
    d = os.path.abspath(out_dir)
    os.makedirs(mesh_dir, exist_ok=True)
    mesh_path = os.path.join(os.path.abspath(mesh_dir), f"icosphere_s{subdiv}.obj")
    if not os.path.exists(mesh_path):
        V, N, F = displaced_icosphere(subdiv, 1234)
        write_indexed_obj(mesh_path, V, N, F)
    with open(base) as f:
        scene = json.load(f)
    rng = np.random.default_rng(seed)
    side = int(np.ceil(np.sqrt(n_instances)))
    spacing = 0.9 / side
    s = 0.4 * spacing
    for i in range(n_instances):
        kind = ["lambertian", "blinn", "thinfilm"][int(rng.integers(0, 3))]
        name = f"m{i}"
        if kind == "lambertian":
            p = os.path.join(d, f"albedo_{i}.csv")
            smooth_random_csv(p, rng)
            scene["materials"].append({"name": name, "type": "lambertian", "albedo": {"val": p}})
        elif kind == "blinn":
            p = os.path.join(d, f"kd_{i}.csv")
            smooth_random_csv(p, rng, 0.05, 0.6)
            alpha = 2 * int(round(np.exp(rng.uniform(np.log(8), np.log(2048))) / 2))
            scene["materials"].append({"name": name, "type": "blinn", "Kd": {"val": p},
                                       "Ks": {"val": float(rng.uniform(0.2, 0.5))}, "glossiness": alpha})
        else:
            alpha = 2 * int(round(np.exp(rng.uniform(np.log(8), np.log(2048))) / 2))
            scene["materials"].append({"name": name, "type": "thinfilm",
                                       "film_ior": {"val": float(rng.uniform(1.33, 1.6))},
                                       "base_ior": {"val": 1.5}, "glossiness": alpha,
                                       "thickness": float(rng.uniform(200, 800))})
        gx, gy = i % side, i // side
        scene["objects"].append({"name": f"inst{i}", "type": "trimesh", "material": name,
                                 "source": mesh_path,
                                 "transform": {"scale": [s, s, s],
                                               "rotate": {"axis": [0, 0, 1],
                                                          "degrees": float(rng.uniform(0, 360))},
                                               "translate": [0.05 + (gx + 0.5) * spacing,
                                                             0.05 + (gy + 0.5) * spacing, s]}})
    with open(base, "w") as f:
        json.dump(scene, f, indent=1)
    return base


def batch_jobs(n_jobs=64, seed=2024):
    """The batched workload: per job an instance count U[1,128], an
    icosphere subdivision from {5, 6, 7} (20K-328K triangles per instance),
    a square resolution from {128, 256, 512, 1024}, spp log-uniform in
    [4, 256] and bounces U[4, 32]; p = 0.8.  Returns a list of dicts."""
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n_jobs):
        jobs.append(dict(n_instances=int(rng.integers(1, 129)), subdiv=int(rng.integers(5, 8)),
                         width=int(rng.choice([128, 256, 512, 1024])),
                         spp=int(round(np.exp(rng.uniform(np.log(4), np.log(256))))),
                         max_scatterings=int(rng.integers(4, 33)), sample_p=0.8, seed=1000 + k))
    return jobs


def uv_sphere(n_lon=24, n_lat=14):
    """Unit UV sphere: n_lon * (n_lat - 2) * 2 + 2 * n_lon triangles with
    outward vertex normals; returns V, N, F (0-based)."""
    V = [(0.0, 0.0, 1.0)]
    for i in range(1, n_lat):
        th = np.pi * i / n_lat
        for j in range(n_lon):
            ph = 2 * np.pi * j / n_lon
            V.append((np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)))
    V.append((0.0, 0.0, -1.0))
    V = np.asarray(V, np.float64)
    F = []
    for j in range(n_lon):
        F.append((0, 1 + j, 1 + (j + 1) % n_lon))
    for i in range(n_lat - 2):
        r0, r1 = 1 + i * n_lon, 1 + (i + 1) * n_lon
        for j in range(n_lon):
            a, b = r0 + j, r0 + (j + 1) % n_lon
            c, d = r1 + j, r1 + (j + 1) % n_lon
            F.append((a, c, d))
            F.append((a, d, b))
    last = len(V) - 1
    r0 = 1 + (n_lat - 2) * n_lon
    for j in range(n_lon):
        F.append((r0 + j, last, r0 + (j + 1) % n_lon))
    return V, V.copy(), np.asarray(F, np.int64)


ALBEDO_BINS = 32


def albedo_wavelengths(n=ALBEDO_BINS):
    """The sample wavelengths of an n-sample albedo on 400-720 nm, as
    written to (and read back from) its CSV."""
    return [float("%.6f" % x) for x in np.linspace(400.0, 720.0, n)]


def albedo_csv(path, values):
    """n-sample albedo spectrum on 400-720 nm (the reference's spectral
    range), read by the reference's box-average loader (cg.hpp:252-272)."""
    lam = albedo_wavelengths(len(values))
    with open(path, "w") as f:
        for l, v in zip(lam, values):
            f.write("%.6f,%.6f\n" % (l, v))


def diff_scene(out_dir, albedo, thickness, width=512, film_ior=1.45, base_ior=1.6, alpha=8, seed=9):
    """The inverse-rendering scene: a ground of G x G thin-film tiles (one
    2-triangle quad object and material per tile, thickness[i, j] nm) under
    64 Lambertian UV spheres (624 triangles each, albedo[k] = 32 samples on
    400-720 nm), lit by two quad lights; about 50K triangles in all.
    Returns the .nls path."""
    os.makedirs(out_dir, exist_ok=True)
    d = os.path.abspath(out_dir)
    albedo = np.asarray(albedo, np.float64)
    thickness = np.asarray(thickness, np.float64)
    G = thickness.shape[0]
    rng = np.random.default_rng(seed)
    tile = os.path.join(d, "tile.obj")
    # the tile quad at z = 1, moved to z = 0 by each tile's transform
    _write_flat_mesh(tile, [[(0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]])
    sph = os.path.join(d, "sphere.obj")
    V, N, F = uv_sphere()
    write_indexed_obj(sph, V, N, F)
    blackbody_csv(os.path.join(d, "bb6500.csv"), 6500.0, 4.0)
    blackbody_csv(os.path.join(d, "bb3500.csv"), 3500.0, 2.5)
    extent = 8.0
    s = extent / G
    materials, objects = [], []
    for i in range(G):
        for j in range(G):
            name = f"film_{i}_{j}"
            materials.append({"name": name, "type": "thinfilm", "glossiness": alpha,
                              "thickness": float(thickness[i, j]), "film_ior": {"val": film_ior},
                              "base_ior": {"val": base_ior}})
            objects.append({"name": f"tile_{i}_{j}", "type": "trimesh", "material": name, "source": tile,
                            "transform": {"scale": [s, s, 1],
                                          "translate": [-extent / 2 + j * s, -extent / 2 + i * s, -1.0]}})
    n_sph = albedo.shape[0]
    side = int(np.ceil(np.sqrt(n_sph)))
    for k in range(n_sph):
        p = os.path.join(d, f"albedo_{k}.csv")
        albedo_csv(p, albedo[k])
        name = f"alb_{k}"
        materials.append({"name": name, "type": "lambertian", "albedo": {"val": p}})
        r = 0.22 + 0.08 * float(rng.uniform())
        gx, gy = k % side, k // side
        objects.append({"name": f"sphere_{k}", "type": "trimesh", "material": name, "source": sph,
                        "transform": {"scale": [r, r, r],
                                      "translate": [(gx - (side - 1) / 2) * extent / side,
                                                    (gy - (side - 1) / 2) * extent / side, r + 0.05]}})
    # the lights' mirror images in the ground fall inside the view, so the
    # thin-film highlights (whose colour the thickness sets) are seen
    lights = [
        {"name": "key", "type": "quaddir", "specular": 2,
         "transform": {"scale": [3.0, 3.0, 1], "rotate": {"axis": [1, 0, 0], "degrees": 180},
                       "translate": [0.0, 3.0, 7.0]},
         "radiance": {"val": os.path.join(d, "bb6500.csv")}},
        {"name": "fill", "type": "quaddir", "specular": 2,
         "transform": {"scale": [2.0, 2.0, 1], "rotate": {"axis": [1, 0, 0], "degrees": 180},
                       "translate": [2.5, 5.0, 6.0]},
         "radiance": {"val": os.path.join(d, "bb3500.csv")}},
    ]
    scene = {"camera": {"pos": [0.0, -7.5, 8.5], "look_at": [0.0, -0.3, 0.0], "up": [0, 0, 1],
                        "fov": 45, "ar": 1.0, "width": width},
             "materials": materials, "objects": objects, "lights": lights}
    path = os.path.join(d, "scene.nls")
    with open(path, "w") as f:
        json.dump(scene, f)
    return path
