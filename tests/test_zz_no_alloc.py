"""lgpu_tonemap_noalloc: the tone map for callers that cannot allocate device
memory when they call the library — for instance an engine whose device
memory is all carved out of pre-sized pools, where a cudaMalloc in the frame
loop would synchronise the device.  It keeps its scratch (partial sums of
log-luminance and the exposure) in a fixed device array inside the library
instead of allocating it.

The test calls it through the C ABI on device buffers, twice in a row on
different images, and checks each result against lgpu_tonemap (the
allocating entry point) within the tolerance of the other tone-map test.
This file is collected last so that a run stopping at the first failure has
run every other test first; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from lambda_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _noalloc(img_dev, w, h, y_mid, torch):
    out_tm = torch.empty_like(img_dev)
    out_24 = torch.empty(img_dev.shape, dtype=torch.uint8, device=img_dev.device)
    rc = L.lib().lgpu_tonemap_noalloc(ctypes.c_void_p(img_dev.data_ptr()), w, h, y_mid,
                                      ctypes.c_void_p(out_tm.data_ptr()),
                                      ctypes.c_void_p(out_24.data_ptr()),
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == L.OK, rc
    return out_tm.cpu().numpy(), out_24.cpu().numpy()


def test_tonemap_noalloc_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    from lambda_b200.renderer import Context
    ctx = Context()
    rng = np.random.default_rng(3)
    for w, h, y_mid in ((37, 23, 0.12), (640, 360, 0.18)):
        # a wide dynamic range, like a rendered image's linear radiance
        img = (rng.lognormal(mean=3.0, sigma=1.5, size=(h, w, 3))).astype(np.float32)
        img[0, 0] = 0.0
        tm_ref, b_ref = ctx.tonemap(img, y_mid)
        dev = torch.from_numpy(img).cuda()
        tm, b = _noalloc(dev, w, h, y_mid, torch)
        assert np.allclose(tm, tm_ref, rtol=1e-4, atol=1e-6)
        assert np.max(np.abs(b.astype(int) - b_ref.astype(int))) <= 1


def test_tonemap_noalloc_rejects_oversized_images():
    lib = L.lib()
    # the size check comes before any device access
    big = 1 << 16
    rc = lib.lgpu_tonemap_noalloc(ctypes.c_void_p(16), big, big, 0.12, ctypes.c_void_p(16), None, None)
    assert rc == L.ERR_TOO_LARGE
    assert lib.lgpu_tonemap_noalloc(None, 4, 4, 0.12, None, None, None) == L.ERR_INVALID_ARGUMENT
