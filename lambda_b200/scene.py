"""Scene model and .nls loader — the Python host's mirror of the reference's
nl::cg::scene (cg.hpp:766-1180) and nl::cg::load (cg.hpp:1993-2474).

Every float the loader produces is computed with single-precision operations
in the reference's order (numpy float32 scalars, libm's cosf/sinf/tanf, libc
strtof for CSV fields, fast_obj's own decimal parser for OBJ files), so a
scene loaded here flattens to the same arrays as the reference loader's
scene flattened by the C++ drop-in (lambda_b200/host/lgpu_flatten.hpp).

Quirks of the reference that are kept because the renderer's output depends
on them:
  * mesh bounds include fast_obj's dummy vertex (0,0,0) (cg.hpp:2218-2229);
  * the camera x axis is up^z without normalisation (cg.hpp:2063-2065);
  * a light's emitter material is shared by name "emitter_<radiance>"
    (cg.hpp:2085-2091, 2109-2115);
  * a Blinn spectrum given as a bare number (no "val") loads as zero
    (cg.hpp:2366-2370);
  * group transforms are not applied to their children (cg.hpp:2318).
"""
import ctypes
import json
import math
import os

import numpy as np

from . import _lib as L

F32 = np.float32
_libm = ctypes.CDLL("libm.so.6")
_libc = ctypes.CDLL("libc.so.6")
for _n in ("cosf", "sinf", "tanf"):
    getattr(_libm, _n).restype = ctypes.c_float
    getattr(_libm, _n).argtypes = [ctypes.c_float]
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]

PI = F32(3.14159274101257324)  # std::numbers::pi_v<float>
FLT_MAX = F32(np.finfo(np.float32).max)


def cosf(x):
    return F32(_libm.cosf(float(x)))


def sinf(x):
    return F32(_libm.sinf(float(x)))


def tanf(x):
    return F32(_libm.tanf(float(x)))


def stof(s):
    """std::stof: strtof of the string (leading whitespace allowed)."""
    return F32(_libc.strtof(s.encode(), None))


def nl_min(a, b):
    return a if a <= b else b


def nl_max(a, b):
    return a if a >= b else b


# ---- spectra -----------------------------------------------------------------

class SpectralConfig:
    """coefficientλ<n> on [inf, sup] and the hero count.  The reference
    compiles in n=80, [400, 720] nm, 16 hero wavelengths (cg.hpp:40-41,
    244-245)."""

    def __init__(self, n_bins=80, lambda_inf=400.0, lambda_sup=720.0, hero_k=16):
        self.n_bins = int(n_bins)
        self.inf = F32(lambda_inf)
        self.sup = F32(lambda_sup)
        self.hero_k = int(hero_k)
        self.delta = F32(F32(self.sup - self.inf) / F32(self.n_bins - 1))

    def key(self):
        return (self.n_bins, float(self.inf), float(self.sup))


REFERENCE_SPECTRAL = SpectralConfig()


def coef_from_samples(l, v, cfg):
    """coefficientλ(sampledλ) (cg.hpp:252-272): box average of the piecewise
    linear samples (l sorted) over each bin [inf+iΔ, inf+(i+1)Δ)."""
    n = cfg.n_bins
    D = cfg.delta
    out = np.zeros(n, np.float32)
    l = [F32(x) for x in l]
    v = [F32(x) for x in v]
    size = len(l)
    j = 0
    half = F32(0.5)
    for i in range(n):
        l0 = F32(cfg.inf + F32(F32(i) * D))
        l1 = F32(l0 + D)
        s = F32(0.0)
        while j + 1 < size and l[j + 1] <= l0:
            j += 1
        k = j
        while k + 1 < size and l[k] < l1:
            seg0 = nl_max(l0, l[k])
            seg1 = nl_min(l1, l[k + 1])
            seg = F32(seg1 - seg0)
            if seg > 0:
                s = F32(s + F32(F32(half * F32(v[k] + v[k + 1])) * seg))
            k += 1
        out[i] = F32(s / D)
    return out


def coef_dot(a, b, cfg):
    """coefficientλ::operator| (cg.hpp:283-288)."""
    s = F32(0.0)
    for x, y in zip(a, b):
        s = F32(s + F32(x * y))
    return F32(s * cfg.delta)


def read_csv_spectrum(path):
    """sampledλ(fpath) (cg.hpp:205-219): 'λ,value' rows."""
    ls, vs = [], []
    with open(path) as f:
        for line in f.read().split("\n"):
            if line == "":
                continue
            parts = line.split(",")
            ls.append(stof(parts[0]))
            vs.append(stof(parts[1] if len(parts) > 1 else ""))
    return ls, vs


_TABLE_CACHE = {}


def cie_tables(cfg):
    """(cmf_x, cmf_y, cmf_z, bt709_r, bt709_g, bt709_b) as coefficient
    spectra of cfg, from the tables the reference loads at start-up
    (cg.hpp:329-337)."""
    key = cfg.key()
    if key in _TABLE_CACHE:
        return _TABLE_CACHE[key]
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "data", "cie_tables.json")) as f:
        d = json.load(f)
    out = []
    for axis in "xyz":
        rows = d[f"cmf_{axis}"]
        out.append(coef_from_samples([stof(r[0]) for r in rows], [stof(r[1]) for r in rows], cfg))
    b = d["bt709_basis"]
    lmin, lstep = F32(b["lambda_min"]), F32(b["lambda_step"])
    ls = [F32(lmin + F32(F32(n) * lstep)) for n in range(len(b["rows"]))]
    for c in range(3):
        out.append(coef_from_samples(ls, [stof(r[c]) for r in b["rows"]], cfg))
    _TABLE_CACHE[key] = tuple(out)
    return _TABLE_CACHE[key]


# ---- algebra (bra.hpp) ---------------------------------------------------------

def v3(x):
    return [F32(x[0]), F32(x[1]), F32(x[2])]


def dot3(a, b):
    return F32(F32(F32(a[0] * b[0]) + F32(a[1] * b[1])) + F32(a[2] * b[2]))


def cross3(x, y):
    return [F32(F32(x[1] * y[2]) - F32(x[2] * y[1])), F32(F32(x[2] * y[0]) - F32(x[0] * y[2])),
            F32(F32(x[0] * y[1]) - F32(x[1] * y[0]))]


def len2(a):
    s = F32(0.0)
    for x in a:
        s = F32(s + F32(x * x))
    return s


def l2(a):
    return F32(np.sqrt(len2(a)))


def normalized(a):
    ln = l2(a)
    return [F32(x / ln) for x in a]


def sub3(a, b):
    return [F32(a[i] - b[i]) for i in range(3)]


def mat4_mul(A, B):
    """ℝnxm * ℝnxm (bra.hpp:310-322), row-major 4x4."""
    out = np.zeros(16, np.float32)
    for i in range(4):
        for j in range(4):
            s = F32(0.0)
            for k in range(4):
                s = F32(s + F32(A[i * 4 + k] * B[k * 4 + j]))
            out[i * 4 + j] = s
    return out


class Transform:
    """nl::cg::transform (cg.hpp:422-488)."""

    def __init__(self, M=None, M_inv=None):
        self.M = np.eye(4, dtype=np.float32).reshape(16) if M is None else np.asarray(M, np.float32)
        self.M_inv = (np.eye(4, dtype=np.float32).reshape(16) if M_inv is None
                      else np.asarray(M_inv, np.float32))

    @staticmethod
    def scale(x):
        T = Transform()
        for i in range(3):
            T.M[i * 5] = F32(x[i])
            T.M_inv[i * 5] = F32(F32(1.0) / F32(x[i]))
        return T

    @staticmethod
    def rotate(axis, degrees):
        u = normalized(v3(axis))
        th = F32(F32(F32(degrees) * PI) / F32(180.0))
        c = cosf(th)
        s = sinf(th)
        o = F32(F32(1.0) - c)
        T = Transform()
        M, Mi = T.M, T.M_inv

        def p(a, b):
            return F32(F32(o * u[a]) * u[b])

        M[0] = F32(c + p(0, 0))
        M[1] = F32(p(0, 1) + F32(s * u[2]))
        M[2] = F32(p(0, 2) - F32(s * u[1]))
        M[4] = F32(p(1, 0) - F32(s * u[2]))
        M[5] = F32(c + p(1, 1))
        M[6] = F32(p(1, 2) + F32(s * u[0]))
        M[8] = F32(p(2, 0) + F32(s * u[1]))
        M[9] = F32(p(2, 1) - F32(s * u[0]))
        M[10] = F32(c + p(2, 2))
        Mi[0] = F32(c + p(0, 0))
        Mi[1] = F32(p(0, 1) - F32(s * u[2]))
        Mi[2] = F32(p(0, 2) + F32(s * u[1]))
        Mi[4] = F32(p(1, 0) + F32(s * u[2]))
        Mi[5] = F32(c + p(1, 1))
        Mi[6] = F32(p(1, 2) - F32(s * u[0]))
        Mi[8] = F32(p(2, 0) - F32(s * u[1]))
        Mi[9] = F32(p(2, 1) + F32(s * u[0]))
        Mi[10] = F32(c + p(2, 2))
        return T

    @staticmethod
    def translate(x):
        T = Transform()
        for i in range(3):
            T.M[i * 4 + 3] = F32(x[i])
            T.M_inv[i * 4 + 3] = F32(-F32(x[i]))
        return T

    def then(self, T2):
        """operator<< (cg.hpp:491-497): self first, then T2."""
        return Transform(mat4_mul(T2.M, self.M), mat4_mul(self.M_inv, T2.M_inv))

    def column(self, j):
        return [self.M[i * 4 + j] for i in range(3)]

    def pos(self):
        return self.column(3)


def load_transform(j):
    """loadTransform (cg.hpp:2004-2021)."""
    sc = [F32(x) for x in j["scale"]] if "scale" in j else [F32(1.0)] * 3
    tr = [F32(x) for x in j["translate"]] if "translate" in j else [F32(0.0)] * 3
    try:
        rot = j["rotate"]
        axis = [F32(x) for x in rot["axis"]]
        deg = F32(rot["degrees"])
    except (KeyError, TypeError, IndexError):
        axis, deg = [F32(0), F32(0), F32(1)], F32(0)
    return Transform.scale(sc).then(Transform.rotate(axis, deg)).then(Transform.translate(tr))


# ---- scene structures --------------------------------------------------------

class Camera:
    """nl::cg::camera (cg.hpp:1151-1165) as loadCamera sets it
    (cg.hpp:2039-2069)."""

    def __init__(self, pos, look_at, up, width, fov, ar=1.77778, dof=0.0, f=1.0):
        self.pos = v3(pos)
        self.fov = F32(fov)
        self.dof = F32(dof)
        self.D = F32(f)
        self.width = int(width)
        self.height = int(math.ceil(F32(F32(self.width) / F32(ar))))
        z = normalized(sub3(self.pos, v3(look_at)))
        x = cross3(v3(up), z)
        y = cross3(z, x)
        self.base = (x, y, z)
        half = F32(F32(0.5) * F32(F32(self.fov * PI) / F32(180.0)))
        self.delta = F32(F32(F32(F32(2.0) * self.D) * tanf(half)) / F32(self.height))
        self.h = F32(self.delta * F32(self.height))
        self.w = F32(self.delta * F32(self.width))


class Material:
    """One entry of list<Material>: kind in lambertian, blinn, thinfilm,
    microfacet, emitter, diremitter (cg.hpp:1084-1085)."""

    def __init__(self, kind, name, **kw):
        self.kind = kind
        self.name = name
        self.__dict__.update(kw)


class Object:
    def __init__(self, kind, name, T, mat, obj, mesh=0):
        self.kind, self.name, self.T, self.mat, self.obj, self.mesh = kind, name, T, mat, obj, mesh


class LightDef:
    def __init__(self, kind, name, **kw):
        self.kind = kind
        self.name = name
        self.__dict__.update(kw)


class TriMeshData:
    """trimeshdata (cg.hpp:766-820): positions and normals with fast_obj's
    dummy element at index 0, faces as (V0,V1,V2,N0,N1,N2), face normals,
    bounds and the reference-layout wide BVH."""

    def __init__(self, name, V, N, F, cfg=None):
        self.name = name
        self.V = np.ascontiguousarray(V, np.float32).reshape(-1, 3)
        self.N = np.ascontiguousarray(N, np.float32).reshape(-1, 3)
        self.F = np.ascontiguousarray(F, np.uint32).reshape(-1, 6)
        # bounds over every position, the dummy included (cg.hpp:2215-2229)
        self.bounds = np.concatenate([self.V.min(axis=0), self.V.max(axis=0)]).astype(np.float32)
        self.GN = face_normals(self.V, self.F)
        self.build_bvh()

    def build_bvh(self):
        """trimeshdata::buildBVH (cg.hpp:792) through the library's
        restatement of bvh::build, and the mesh's traversal tree
        (lgpu_build_traversal_bvh: the tree the renders' instance-BVH
        traversal enters), both at load as the reference builds its tree.
        The traversal tree is skipped for meshes with non-finite vertices
        (the upload then traverses the reference's tree)."""
        self.nodes, self.bbs, self.prim_idxs = self._tree("lgpu_build_bvh")
        try:
            self.trav_nodes, self.trav_bbs, self.trav_prim_idxs = self._tree("lgpu_build_traversal_bvh")
        except L.LgpuError:
            self.trav_nodes = self.trav_bbs = self.trav_prim_idxs = None

    def _tree(self, fn):
        nf = self.F.shape[0]
        nodes = np.zeros(4 * nf + 4, np.uint32)
        bbs = np.zeros(96 * nf + 96, np.float32)
        prims = np.zeros(nf + 1, np.uint32)
        nn, nb, npi = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        rc = getattr(L.lib(), fn)(self.V.ctypes.data, self.V.shape[0], self.F.ctypes.data, 6, nf,
                                  nodes.ctypes.data, ctypes.byref(nn), bbs.ctypes.data,
                                  ctypes.byref(nb), prims.ctypes.data, ctypes.byref(npi))
        if rc != 0:
            raise L.LgpuError(rc, fn + " failed")
        return nodes[:2 * nn.value].copy(), bbs[:48 * nb.value].copy(), prims[:npi.value].copy()


def face_normals(V, F):
    """(e0 ^ e2).normalized() with e0 = V1-V0, e2 = V2-V0 (cg.hpp:2258-2262),
    vectorised with float32 operations in the same order."""
    v0 = V[F[:, 0]]
    v1 = V[F[:, 1]]
    v2 = V[F[:, 2]]
    e0 = v1 - v0
    e2 = v2 - v0
    c = np.empty_like(e0)
    c[:, 0] = e0[:, 1] * e2[:, 2] - e0[:, 2] * e2[:, 1]
    c[:, 1] = e0[:, 2] * e2[:, 0] - e0[:, 0] * e2[:, 2]
    c[:, 2] = e0[:, 0] * e2[:, 1] - e0[:, 1] * e2[:, 0]
    l2v = ((np.float32(0) + c[:, 0] * c[:, 0]) + c[:, 1] * c[:, 1]) + c[:, 2] * c[:, 2]
    ln = np.sqrt(l2v).astype(np.float32)
    return (c / ln[:, None]).astype(np.float32)


# ---- OBJ (fast_obj semantics) ------------------------------------------------------

_POW10_POS = [float("1e%d" % k) for k in range(20)]
_POW10_NEG = [float("1e-%d" % k) for k in range(20)]


def fast_obj_float(tok):
    """fast_obj's parse_float: sign, integer and fraction digits accumulated
    in double precision, num += fra/div, an optional power of ten from its
    table, then (float)."""
    i = 0
    sign = 1.0
    if tok[i:i + 1] == "+":
        i += 1
    elif tok[i:i + 1] == "-":
        sign = -1.0
        i += 1
    num = 0.0
    while i < len(tok) and tok[i].isdigit():
        num = 10.0 * num + float(ord(tok[i]) - 48)
        i += 1
    if i < len(tok) and tok[i] == ".":
        i += 1
    fra, div = 0.0, 1.0
    while i < len(tok) and tok[i].isdigit():
        fra = 10.0 * fra + float(ord(tok[i]) - 48)
        div *= 10.0
        i += 1
    num += fra / div
    if i < len(tok) and tok[i] in "eE":
        i += 1
        table = _POW10_POS
        if i < len(tok) and tok[i] in "+-":
            table = _POW10_NEG if tok[i] == "-" else _POW10_POS
            i += 1
        ev = 0
        while i < len(tok) and tok[i].isdigit():
            ev = 10 * ev + ord(tok[i]) - 48
            i += 1
        num *= 0.0 if ev >= 20 else table[ev]
    return np.float32(sign * num)


def _parse_floats(tokens):
    """fast_obj_float over an array of plain decimal tokens ([-]I.F, no
    exponent), vectorised; tokens with an exponent go through the scalar
    parser."""
    toks = np.asarray(tokens)
    out = np.empty(toks.shape, np.float32)
    if toks.size == 0:
        return out
    flat = toks.reshape(-1)
    res = out.reshape(-1)
    has_exp = np.char.find(flat, "e") >= 0
    has_exp |= np.char.find(flat, "E") >= 0
    neg = np.char.startswith(flat, "-")
    body = np.where(neg | np.char.startswith(flat, "+"), np.char.lstrip(flat, "+-"), flat)
    parts = np.char.partition(body, ".")
    ip = parts[:, 0] if parts.ndim == 2 else parts[..., 0]
    fp = parts[:, 2] if parts.ndim == 2 else parts[..., 2]
    ok = ~has_exp
    ip_f = np.array([float(int(x)) if x else 0.0 for x in ip[ok]], np.float64)
    flen = np.char.str_len(fp[ok])
    fp_f = np.array([float(int(x)) if x else 0.0 for x in fp[ok]], np.float64)
    div = np.array([10.0 ** int(n) for n in flen], np.float64)
    num = ip_f + fp_f / div
    sgn = np.where(neg[ok], -1.0, 1.0)
    res[ok] = (sgn * num).astype(np.float32)
    for k in np.nonzero(has_exp)[0]:
        res[k] = fast_obj_float(str(flat[k]))
    return out


def read_obj(path):
    """Triangle OBJ reader with fast_obj's indexing (1-based, dummy element 0,
    dummy normal (0,0,1)) and its float parser; returns V, N, F for
    TriMeshData."""
    with open(path) as f:
        lines = f.read().split("\n")
    vt, nt, ft = [], [], []
    for line in lines:
        if line.startswith("v "):
            vt.append(line.split()[1:4])
        elif line.startswith("vn "):
            nt.append(line.split()[1:4])
        elif line.startswith("f "):
            t = line.split()[1:]
            if len(t) != 3:
                raise ValueError("the reference loader reads triangles only (cg.hpp:2252)")
            ft.append(t)
    V = np.zeros((len(vt) + 1, 3), np.float32)
    N = np.zeros((len(nt) + 1, 3), np.float32)
    N[0] = (0.0, 0.0, 1.0)
    if vt:
        V[1:] = _parse_floats(np.array(vt))
    if nt:
        N[1:] = _parse_floats(np.array(nt))
    F = np.zeros((len(ft), 6), np.uint32)
    nv, nn = V.shape[0], N.shape[0]
    for r, t in enumerate(ft):
        for k, tok in enumerate(t):
            parts = tok.split("/")
            p = int(parts[0])
            n = int(parts[2]) if len(parts) > 2 and parts[2] else 0
            F[r, k] = p if p > 0 else nv + p
            F[r, 3 + k] = n if n > 0 else (nn + n if n < 0 else 0)
    return V, N, F


def write_obj(path, V, N, F, fmt="%.6f"):
    """Writes positions (without the dummy), normals and 1-based triangle
    faces `f v//n` in a form both fast_obj and read_obj parse identically."""
    with open(path, "w") as f:
        lines = []
        for v in V:
            lines.append("v " + " ".join(fmt % x for x in v))
        for n in N:
            lines.append("vn " + " ".join(fmt % x for x in n))
        for t in F:
            lines.append("f %d//%d %d//%d %d//%d" % (t[0], t[3], t[1], t[4], t[2], t[5]))
        f.write("\n".join(lines) + "\n")


# ---- scene and loader ------------------------------------------------------------

class SceneData:
    """nl::cg::scene (cg.hpp:1167-1180)."""

    def __init__(self, cfg=None):
        self.cfg = cfg or REFERENCE_SPECTRAL
        self.cam = None
        self.objects = []
        self.materials = []
        self.lights = []
        self.meshes = []

    def material_index(self, name):
        for i, m in enumerate(self.materials):
            if m.name == name:
                return i
        return len(self.materials)


def coef_to_string(s):
    """coefficientλ::toString (cg.hpp:321-326)."""
    return "".join("%.2f" % float(x) for x in s)


def load_spectrum(j, cfg, base_dir):
    """loadSpectrum (cg.hpp:2022-2036)."""
    val = j["val"]
    if isinstance(val, str):
        p = val if os.path.isabs(val) else os.path.join(base_dir, val)
        ls, vs = read_csv_spectrum(p)
        s = coef_from_samples(ls, vs, cfg)
    elif isinstance(val, (int, float)) and not isinstance(val, bool):
        s = np.full(cfg.n_bins, F32(val), np.float32)
    else:
        rgb = [F32(x) for x in val]
        r, g, b = cie_tables(cfg)[3:]
        s = ((r * rgb[0]) + (g * rgb[1])) + (b * rgb[2])
        s = s.astype(np.float32)
    mul = F32(j["mult"]) if "mult" in j else F32(1.0)
    return (s * mul).astype(np.float32)


def _opt_spectrum(j, key, default, cfg, base_dir):
    try:
        return load_spectrum(j[key], cfg, base_dir)
    except (KeyError, TypeError):
        return np.full(cfg.n_bins, F32(default), np.float32)


def blinn_init(m, cfg):
    """blinn::init (cg.hpp:931-940)."""
    diff = F32(np.sqrt(coef_dot(m.Kd, m.Kd, cfg)))
    m.w_r = F32(np.sqrt(coef_dot(m.Ks, m.Ks, cfg)))
    m.w_t = F32(np.sqrt(coef_dot(m.Kt, m.Kt, cfg)))
    tot = F32(F32(diff + m.w_r) + m.w_t)
    if not tot > 0:
        raise ValueError(f"blinn material {m.name}: all lobes are zero (assert at cg.hpp:937)")
    m.p_d = F32(diff / tot)
    m.p_spec = F32(F32(m.w_r + m.w_t) / tot)


# parsed meshes shared by every scene loaded in this process, keyed by the
# file's identity (a mesh is read-only once built)
_MESH_CACHE = {}


def _load_mesh(src, path):
    st = os.stat(path)
    key = (src, os.path.abspath(path), st.st_mtime_ns, st.st_size)
    m = _MESH_CACHE.get(key)
    if m is None:
        V, N, F = read_obj(path)
        m = TriMeshData(src, V, N, F)
        _MESH_CACHE[key] = m
    return m


def load_nls(path, cfg=None, base_dir=None):
    """loadNLS (cg.hpp:2455-2470).  Relative file names inside the scene are
    resolved against base_dir (default: the directory the reference binary is
    run from, i.e. the scene file's parent's parent for bin/scenes/*.nls
    layouts, else the scene file's directory)."""
    cfg = cfg or REFERENCE_SPECTRAL
    with open(path) as f:
        j = json.load(f)
    if base_dir is None:
        base_dir = os.path.dirname(os.path.abspath(path))
    sc = SceneData(cfg)
    c = j["camera"]
    sc.cam = Camera(c["pos"], c["look_at"], c["up"], c["width"], c["fov"], c.get("ar", 1.77778),
                    c.get("dof", 0.0), c.get("f", 1.0))
    # materials (cg.hpp:2399-2450)
    for jm in j["materials"]:
        name, kind = jm["name"], jm["type"]
        if kind == "lambertian":
            sc.materials.append(Material("lambertian", name,
                                         albedo=load_spectrum(jm["albedo"], cfg, base_dir)))
        elif kind == "blinn":
            m = Material("blinn", name,
                         Kd=_opt_spectrum(jm, "Kd", 0.0, cfg, base_dir),
                         Ks=_opt_spectrum(jm, "Ks", 0.0, cfg, base_dir),
                         Kt=_opt_spectrum(jm, "Kt", 0.0, cfg, base_dir),
                         Le=_opt_spectrum(jm, "Le", 0.0, cfg, base_dir),
                         ior=_opt_spectrum(jm, "ior", 1.54, cfg, base_dir),
                         alpha=F32(jm.get("glossiness", 1024)))
            blinn_init(m, cfg)
            sc.materials.append(m)
        elif kind == "thinfilm":
            sc.materials.append(Material(
                "thinfilm", name, film_ior=load_spectrum(jm["film_ior"], cfg, base_dir),
                base_ior=_opt_spectrum(jm, "base_ior", 1.54, cfg, base_dir),
                alpha=F32(jm.get("glossiness", 1024)), d=F32(jm.get("thickness", 400))))
        elif kind == "microfacet":
            z = np.zeros(cfg.n_bins, np.float32)
            sc.materials.append(Material("microfacet", name, albedo=z, ior=z.copy()))
    # objects (cg.hpp:2307-2352)
    mesh_index = {}

    def load_objects(lst):
        for jo in lst:
            kind = jo["type"]
            if kind == "group":
                load_objects(jo["children"])
                continue
            T = load_transform(jo["transform"])
            mat = sc.material_index(jo["material"])
            if mat >= len(sc.materials):
                raise ValueError(f"object {jo['name']}: unknown material {jo['material']}")
            if kind in ("sphere", "plane"):
                sc.objects.append(Object(kind, jo["name"], T, mat, len(sc.objects)))
            elif kind == "trimesh":
                src = jo["source"]
                if src not in mesh_index:
                    p = src if os.path.isabs(src) else os.path.join(base_dir, src)
                    mesh_index[src] = len(sc.meshes)
                    sc.meshes.append(_load_mesh(src, p))
                sc.objects.append(Object("trimesh", jo["name"], T, mat, len(sc.objects),
                                         mesh_index[src]))
            else:
                raise ValueError("No corresponding ObjectType.")

    load_objects(j["objects"])
    # lights (cg.hpp:2124-2184)
    for jl in j["lights"]:
        kind, name = jl["type"], jl["name"]
        if kind == "ambient":
            sc.lights.append(LightDef("ambient", name,
                                      radiance=load_spectrum(jl["radiance"], cfg, base_dir)))
        elif kind == "point":
            sc.lights.append(LightDef("point", name,
                                      radiance=load_spectrum(jl["radiant_intensity"], cfg, base_dir),
                                      pos=v3(jl["pos"])))
        elif kind == "direction":
            sc.lights.append(LightDef("direction", name,
                                      radiance=load_spectrum(jl["radiant_intensity"], cfg, base_dir),
                                      dir=v3(jl["dir"])))
        elif kind in ("sphere", "quaddir"):
            rad = load_spectrum(jl["radiance"], cfg, base_dir)
            T = load_transform(jl["transform"])
            mname = "emitter_" + coef_to_string(rad)
            mat = sc.material_index(mname)
            if kind == "sphere":
                if mat == len(sc.materials):
                    sc.materials.append(Material("emitter", mname, radiance=rad))
                size = l2(T.column(0))
                obj = len(sc.objects)
                sc.objects.append(Object("sphere", name, T, mat, obj))
                sc.lights.append(LightDef("sphere", name, radiance=rad, size=size, T=T, obj=obj))
            else:
                spec = F32(jl.get("specular", 1024.0))
                if mat == len(sc.materials):
                    sc.materials.append(Material("diremitter", mname, radiance=rad, specular=spec))
                inv_area = F32(F32(1.0) / F32(l2(T.column(0)) * l2(T.column(1))))
                obj = len(sc.objects)
                sc.objects.append(Object("plane", name, T, mat, obj))
                sc.lights.append(LightDef("quaddir", name, radiance=rad, inv_area=inv_area,
                                          spec=spec, T=T, obj=obj))
        else:
            raise ValueError("No corresponding LightType.")
    return sc


# ---- flattening to the C ABI -------------------------------------------------------

_MAT_CODE = {"lambertian": L.MAT_LAMBERTIAN, "blinn": L.MAT_BLINN, "thinfilm": L.MAT_THINFILM,
             "microfacet": L.MAT_MICROFACET, "emitter": L.MAT_EMITTER,
             "diremitter": L.MAT_DIREMITTER}
_OBJ_CODE = {"sphere": L.OBJ_SPHERE, "plane": L.OBJ_PLANE, "trimesh": L.OBJ_TRIMESH}
_LIGHT_CODE = {"ambient": L.LIGHT_AMBIENT, "point": L.LIGHT_POINT, "direction": L.LIGHT_DIR,
               "sphere": L.LIGHT_SPHERE, "quaddir": L.LIGHT_QUADDIR}


def _fp(a):
    return a.ctypes.data_as(L.c_float_p)


def _up(a):
    return a.ctypes.data_as(L.c_uint32_p)


class FlatScene:
    """The scene as one lgpu_scene; owns every array it points to."""

    def __init__(self, sc):
        cfg = sc.cfg
        self.sc = sc
        spectra = []

        def add(s):
            spectra.append(np.asarray(s, np.float32))
            return len(spectra) - 1

        nm = len(sc.materials)
        self.materials = (L.Material * max(nm, 1))()
        for i, m in enumerate(sc.materials):
            d = self.materials[i]
            d.type = _MAT_CODE[m.kind]
            for k in range(5):
                d.spectrum[k] = -1
            if m.kind == "lambertian":
                d.spectrum[0] = add(m.albedo)
            elif m.kind == "blinn":
                for k, s in enumerate((m.Kd, m.Ks, m.Kt, m.Le, m.ior)):
                    d.spectrum[k] = add(s)
                d.alpha, d.p_d, d.p_spec, d.w_r, d.w_t = m.alpha, m.p_d, m.p_spec, m.w_r, m.w_t
            elif m.kind == "thinfilm":
                d.spectrum[0] = add(m.film_ior)
                d.spectrum[1] = add(m.base_ior)
                d.alpha, d.d = m.alpha, m.d
            elif m.kind == "microfacet":
                d.spectrum[0] = add(m.albedo)
                d.spectrum[1] = add(m.ior)
            elif m.kind == "emitter":
                d.spectrum[0] = add(m.radiance)
            elif m.kind == "diremitter":
                d.spectrum[0] = add(m.radiance)
                d.specular = m.specular
        no = len(sc.objects)
        self.objects = (L.Object * max(no, 1))()
        for i, o in enumerate(sc.objects):
            d = self.objects[i]
            d.type = _OBJ_CODE[o.kind]
            d.mat = o.mat
            d.mesh = o.mesh if o.kind == "trimesh" else 0
            d.T.M[:] = [float(x) for x in o.T.M]
            d.T.M_inv[:] = [float(x) for x in o.T.M_inv]
        nl = len(sc.lights)
        self.lights = (L.Light * max(nl, 1))()
        for i, l in enumerate(sc.lights):
            d = self.lights[i]
            d.type = _LIGHT_CODE[l.kind]
            d.spectrum = add(l.radiance)
            if l.kind == "point":
                d.pos[:] = [float(x) for x in l.pos]
            elif l.kind == "direction":
                d.dir[:] = [float(x) for x in l.dir]
            elif l.kind == "sphere":
                d.size = l.size
                d.obj = l.obj
                d.T.M[:] = [float(x) for x in l.T.M]
                d.T.M_inv[:] = [float(x) for x in l.T.M_inv]
            elif l.kind == "quaddir":
                d.inv_area, d.spec, d.obj = l.inv_area, l.spec, l.obj
                d.T.M[:] = [float(x) for x in l.T.M]
                d.T.M_inv[:] = [float(x) for x in l.T.M_inv]
        self.spectra = (np.stack(spectra).astype(np.float32) if spectra
                        else np.zeros((1, cfg.n_bins), np.float32))
        self.spectra = np.ascontiguousarray(self.spectra)
        self.meshes = (L.Mesh * max(len(sc.meshes), 1))()
        for i, m in enumerate(sc.meshes):
            d = self.meshes[i]
            d.n_positions, d.n_normals, d.n_faces, d.f_stride = (m.V.shape[0], m.N.shape[0],
                                                                m.F.shape[0], 6)
            d.V, d.N, d.F, d.GN = _fp(m.V), _fp(m.N), _up(m.F), _fp(m.GN)
            d.bounds[:] = [float(x) for x in m.bounds]
            d.n_nodes, d.n_bbs, d.n_prim_idxs = (m.nodes.size // 2, m.bbs.size // 48,
                                                 m.prim_idxs.size)
            d.nodes, d.bbs, d.prim_idxs = _up(m.nodes), _fp(m.bbs), _up(m.prim_idxs)
            if getattr(m, "trav_nodes", None) is not None:
                d.n_trav_nodes, d.n_trav_bbs, d.n_trav_prim_idxs = (m.trav_nodes.size // 2,
                                                                    m.trav_bbs.size // 48, m.trav_prim_idxs.size)
                d.trav_nodes, d.trav_bbs = _up(m.trav_nodes), _fp(m.trav_bbs)
                d.trav_prim_idxs = _up(m.trav_prim_idxs)
        cmf = cie_tables(cfg)
        self.cmf = [np.ascontiguousarray(cmf[i]) for i in range(3)]
        s = L.Scene()
        cam = sc.cam
        s.cam.base_x[:] = [float(x) for x in cam.base[0]]
        s.cam.base_y[:] = [float(x) for x in cam.base[1]]
        s.cam.base_z[:] = [float(x) for x in cam.base[2]]
        s.cam.pos[:] = [float(x) for x in cam.pos]
        s.cam.fov, s.cam.dof, s.cam.D = cam.fov, cam.dof, cam.D
        s.cam.delta, s.cam.h, s.cam.w = cam.delta, cam.h, cam.w
        s.cam.width, s.cam.height = cam.width, cam.height
        s.spec.n_bins, s.spec.hero_k = cfg.n_bins, cfg.hero_k
        s.spec.lambda_inf, s.spec.lambda_sup = cfg.inf, cfg.sup
        s.spec.cmf_x, s.spec.cmf_y, s.spec.cmf_z = (_fp(self.cmf[0]), _fp(self.cmf[1]),
                                                    _fp(self.cmf[2]))
        s.n_objects, s.n_materials, s.n_lights = no, nm, nl
        s.n_meshes, s.n_spectra = len(sc.meshes), len(spectra)
        s.objects = ctypes.cast(self.objects, ctypes.POINTER(L.Object))
        s.materials = ctypes.cast(self.materials, ctypes.POINTER(L.Material))
        s.lights = ctypes.cast(self.lights, ctypes.POINTER(L.Light))
        s.meshes = ctypes.cast(self.meshes, ctypes.POINTER(L.Mesh))
        s.spectra = _fp(self.spectra)
        self.scene = s

    def ptr(self):
        return ctypes.pointer(self.scene)


def flatten(sc):
    return FlatScene(sc)
