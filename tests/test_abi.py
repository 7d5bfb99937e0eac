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
    assert ctypes.sizeof(L.Mesh) == 112
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
