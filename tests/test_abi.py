"""The C ABI library loads and exports every entry point of
include/lambda_gpu.h; the host-only entry points work without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from lambda_b200 import _lib as L

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(REPO, "include", "lambda_gpu.h")).read()
    return sorted(set(re.findall(r"\b(lgpu_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_symbols()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(L.SIGNATURES), set(names) - set(L.SIGNATURES)


def test_struct_sizes_match_c():
    # sizes of the C structs on x86-64 (include/lambda_gpu.h)
    assert ctypes.sizeof(L.Camera) == 88
    assert ctypes.sizeof(L.Spectral) == 40
    assert ctypes.sizeof(L.Material) == 52
    assert ctypes.sizeof(L.Object) == 144
    assert ctypes.sizeof(L.Light) == 176
    assert ctypes.sizeof(L.Mesh) == 152
    assert ctypes.sizeof(L.Scene) == 192
    assert ctypes.sizeof(L.RenderParams) == 32
    assert ctypes.sizeof(L.Hit) == 56
    assert ctypes.sizeof(L.Job) == 64
    assert L.PROBE_DTYPE.itemsize == 180
    assert L.PROBE_RESULT_DTYPE.itemsize == 96


def test_errors_without_arguments():
    lib = L.lib()
    assert lib.lgpu_create(0, None) == L.ERR_INVALID_ARGUMENT
    assert lib.lgpu_upload_scene(None, None) == L.ERR_INVALID_ARGUMENT
    assert lib.lgpu_build_bvh(None, 0, None, 0, 0, None, None, None, None, None, None) == L.ERR_INVALID_ARGUMENT
    lib.lgpu_destroy(None)
    assert lib.lgpu_last_error(None) == b"no context"


def test_build_bvh_small_meshes():
    """bvh::build on 1..40 triangles: node/prim invariants of the layout."""
    lib = L.lib()
    rng = np.random.default_rng(0)
    for nf in (1, 2, 4, 5, 9, 40):
        V = np.concatenate([np.zeros((1, 3)), rng.uniform(-1, 1, (3 * nf, 3))]).astype(np.float32)
        F = np.zeros((nf, 6), np.uint32)
        F[:, :3] = np.arange(1, 3 * nf + 1).reshape(nf, 3)
        nodes = np.zeros(4 * nf + 4, np.uint32)
        bbs = np.zeros(96 * nf + 96, np.float32)
        prims = np.zeros(nf + 1, np.uint32)
        nn, nb, npi = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        rc = lib.lgpu_build_bvh(V.ctypes.data, V.shape[0], F.ctypes.data, 6, nf, nodes.ctypes.data,
                                ctypes.byref(nn), bbs.ctypes.data, ctypes.byref(nb), prims.ctypes.data,
                                ctypes.byref(npi))
        assert rc == 0
        assert npi.value == nf and sorted(prims[:nf]) == list(range(nf))
        data = nodes[1:2 * nn.value:2]
        leaf = (data & 1) == 1
        assert leaf[0] == (nf <= 4)
        # every leaf holds 1..4 primitives; leaves partition prim_idxs
        cnt = ((data & 0xE) >> 1) + 1
        assert np.all(cnt[leaf] <= 4) and cnt[leaf].sum() == nf


def _traversal_tree(lib, V, F):
    nf = F.shape[0]
    nodes = np.zeros(4 * nf + 4, np.uint32)
    bbs = np.zeros(96 * nf + 96, np.float32)
    prims = np.zeros(nf + 1, np.uint32)
    nn, nb, npi = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    rc = lib.lgpu_build_traversal_bvh(V.ctypes.data, V.shape[0], F.ctypes.data, F.shape[1], nf,
                                      nodes.ctypes.data, ctypes.byref(nn), bbs.ctypes.data, ctypes.byref(nb),
                                      prims.ctypes.data, ctypes.byref(npi))
    return rc, nodes[:2 * nn.value], bbs[:48 * nb.value].reshape(-1, 2, 3, 8), prims[:npi.value]


@pytest.mark.parametrize("nf", [1, 2, 3, 9, 40, 1000, 40000])
def test_traversal_tree_structure(nf):
    """lgpu_build_traversal_bvh: the reference's layout, every face in
    exactly one leaf of at most 2, child boxes enclosing their subtrees'
    faces, breadth-first numbering, and the array bounds of lgpu_build_bvh
    (40,000 faces: the worker threads build it)."""
    lib = L.lib()
    rng = np.random.default_rng(nf)
    # a triangle soup with shared vertices: small triangles around random centres
    c = rng.uniform(-1, 1, (nf, 3))
    V = np.concatenate([np.zeros((1, 3)), (c[:, None, :] + rng.normal(0, 0.02, (nf, 3, 3))).reshape(-1, 3)])
    V = V.astype(np.float32)
    F = np.zeros((nf, 6), np.uint32)
    F[:, :3] = np.arange(1, 3 * nf + 1).reshape(nf, 3)
    rc, nodes, bbs, prims = _traversal_tree(lib, V, F)
    assert rc == 0
    n = nodes.size // 2
    assert n <= 2 * nf and bbs.shape[0] <= 2 * nf
    assert sorted(prims.tolist()) == list(range(nf))
    data = nodes[1::2]
    leaf = (data & 1) == 1
    first = data >> 4
    cnt = ((data >> 1) & 7) + 1
    tri_lo = V[F[:, :3]].min(axis=1)
    tri_hi = V[F[:, :3]].max(axis=1)
    # faces below each node, children after their parent
    below = [None] * n
    for q in range(n - 1, -1, -1):
        if leaf[q]:
            assert nodes[2 * q] == 0xFFFFFFFF and cnt[q] <= 2
            below[q] = prims[first[q]:first[q] + cnt[q]]
        else:
            assert cnt[q] >= 2 and first[q] > q and first[q] + cnt[q] <= n
            below[q] = np.concatenate([below[first[q] + k] for k in range(cnt[q])])
            rec = bbs[nodes[2 * q]]
            for k in range(8):
                if k < cnt[q]:
                    f = below[first[q] + k]
                    assert np.all(rec[0, :, k] <= tri_lo[f].min(axis=0))
                    assert np.all(rec[1, :, k] >= tri_hi[f].max(axis=0))
                else:
                    assert np.all(rec[0, :, k] == np.float32(1e30)) and np.all(rec[1, :, k] == np.float32(-1e30))
    assert sorted(below[0].tolist()) == list(range(nf))
    # leaves are consecutive in breadth-first order
    assert np.array_equal(np.sort(first[leaf]), np.cumsum(np.concatenate([[0], cnt[leaf][:-1]])))


def test_traversal_tree_rejects_bad_input():
    lib = L.lib()
    V = np.zeros((4, 3), np.float32)
    V[1:] = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    F = np.array([[1, 2, 3, 0, 0, 0]], np.uint32)
    assert _traversal_tree(lib, V, F)[0] == 0
    F[0, 2] = 9  # vertex index out of range
    assert _traversal_tree(lib, V, F)[0] == L.ERR_INVALID_ARGUMENT
    F[0, 2] = 3
    V[2, 0] = np.nan
    assert _traversal_tree(lib, V, F)[0] == L.ERR_INVALID_ARGUMENT


def test_no_device_here_is_reported():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = L.lib()
    h = ctypes.c_void_p()
    assert lib.lgpu_create(0, ctypes.byref(h)) == L.ERR_NO_DEVICE


def test_abi_version_matches_header():
    src = open(os.path.join(REPO, "include", "lambda_gpu.h")).read()
    v = int(re.search(r"#define LGPU_ABI_VERSION (\d+)", src).group(1))
    assert L.lib().lgpu_abi_version() == v
