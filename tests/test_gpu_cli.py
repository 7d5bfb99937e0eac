"""The reference's own `lambda` CLI with Renderer::render replaced by the
C-ABI drop-in (lambda_b200/host/renderer_gpu.cpp, built by
lambda_b200/host/Makefile): it renders a scene file end to end and its raw
PNG equals the 8-bit encode of the Python host's render of the same scene
with the same settings and seed."""
import json
import os
import shutil
import struct
import subprocess
import zlib

import numpy as np
import pytest

from lambda_b200 import synth
from lambda_b200.renderer import Context, Rendering
from lambda_b200.scene import load_nls

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "lambda_b200", "host", "_build", "lambda")


def read_png_rgb(path):
    """A non-interlaced PNG (lodepng picks the smallest colour type: grey,
    RGB, palette, with or without alpha) -> (h, w, 3) uint8."""
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, plte = 8, b"", None
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if kind == b"IHDR":
            w, h, depth, ctype, _, _, interlace = struct.unpack(">IIBBBBB", body[:13])
            assert interlace == 0
        elif kind == b"PLTE":
            plte = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    channels = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    bits = channels * depth
    stride = (w * bits + 7) // 8
    bpp = max(1, bits // 8)
    raw = zlib.decompress(idat)
    rows = np.zeros((h, stride), np.uint8)
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        f = raw[y * (stride + 1)]
        row = np.frombuffer(raw, np.uint8, stride, y * (stride + 1) + 1).astype(np.int32)
        cur = np.zeros(stride, np.int32)
        for x in range(stride):
            a = cur[x - bpp] if x >= bpp else 0
            b = prev[x]
            c = prev[x - bpp] if x >= bpp else 0
            if f == 0:
                p = 0
            elif f == 1:
                p = a
            elif f == 2:
                p = b
            elif f == 3:
                p = (a + b) // 2
            else:
                pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                p = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
            cur[x] = (row[x] + p) & 255
        rows[y] = cur
        prev = cur
    if depth < 8:  # packed palette or grey indices
        vals = np.unpackbits(rows, axis=1).reshape(h, -1, depth)[:, :w]
        vals = (vals * (1 << np.arange(depth - 1, -1, -1))).sum(axis=2)
    else:
        assert depth == 8
        vals = rows.reshape(h, w, channels)
    if ctype == 3:
        return plte[vals.reshape(h, w)]
    if ctype in (0, 4):
        # grey below 8 bits is scaled to the full byte range
        g = vals * (255 // ((1 << depth) - 1)) if depth < 8 else vals[..., 0]
        return np.repeat(g[..., None], 3, axis=2).astype(np.uint8)
    return vals[..., :3].astype(np.uint8)


def cmf_files(dst):
    """The CMF tables the reference reads at start-up (cg.hpp:329-337),
    written back from the verbatim entries in lambda_b200/data."""
    d = json.load(open(os.path.join(REPO, "lambda_b200", "data", "cie_tables.json")))
    os.makedirs(dst, exist_ok=True)
    for axis in "xyz":
        with open(os.path.join(dst, "xyz_%s.csv" % axis), "w") as f:
            f.write("".join("%s,%s\n" % (a, b) for a, b in d["cmf_" + axis]))
    with open(os.path.join(dst, "cie1931-basis-bt709-380+5+780.csv"), "w") as f:
        f.write("".join(",".join(r) + "\n" for r in d["bt709_basis"]["rows"]))


@pytest.mark.gpu
def test_reference_cli_renders_on_the_gpu(tmp_path):
    if not os.path.exists(CLI):
        pytest.skip("the CLI was not built (make -C lambda_b200/host needs the reference sources)")
    root = tmp_path / "root"
    cmf_files(str(root / "lib" / "numli" / "data"))
    bin_dir = root / "bin"
    (bin_dir / "scenes").mkdir(parents=True)
    (bin_dir / "render").mkdir()
    nls = synth.mixed(str(tmp_path / "mixed_cli"), width=48)
    shutil.copy(nls, bin_dir / "scenes" / "mixed.nls")
    r = subprocess.run([CLI, "scenes/mixed.nls", "-s", "16", "-b", "8", "-p", "0.8"], cwd=str(bin_dir),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = read_png_rgb(str(bin_dir / "render" / "mixed-16spp-8b-0.80p-raw.png"))
    ctx = Context()
    ctx.upload(load_nls(nls))
    img = ctx.render(16, 8, 0.8, seed=0)
    assert np.array_equal(raw, Rendering(img).rgb24())
    # the tone-mapped PNG: the reference's own toneMap (CPU) of this image
    # (the CLI is built with FMA contraction, the oracle without: bytes
    # agree to 1)
    from oracle import refharness
    tm = np.zeros_like(img)
    b24 = np.zeros(img.shape, np.uint8)
    refharness.RefScene(nls).L.ref_tonemap(img.ctypes.data, img.shape[1], img.shape[0], 0.12, tm.ctypes.data,
                                           b24.ctypes.data)
    mapped = read_png_rgb(str(bin_dir / "render" / "mixed-16spp-8b-0.80p.png"))
    assert np.max(np.abs(mapped.astype(int) - b24.astype(int))) <= 1
    assert len(np.unique(mapped.reshape(-1, 3), axis=0)) > 50


def test_reference_cli_fails_loudly_without_a_device(tmp_path):
    """Without a CUDA device the drop-in render raises (the reference's CLI
    does not catch it): no silent CPU fallback."""
    if not os.path.exists(CLI):
        pytest.skip("the CLI was not built (make -C lambda_b200/host needs the reference sources)")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    root = tmp_path / "root"
    cmf_files(str(root / "lib" / "numli" / "data"))
    bin_dir = root / "bin"
    (bin_dir / "scenes").mkdir(parents=True)
    (bin_dir / "render").mkdir()
    nls = synth.mixed(str(tmp_path / "mixed_cli"), width=16)
    shutil.copy(nls, bin_dir / "scenes" / "mixed.nls")
    r = subprocess.run([CLI, "scenes/mixed.nls", "-s", "1"], cwd=str(bin_dir), capture_output=True, text=True,
                       timeout=300)
    assert r.returncode != 0
    assert "no CUDA device" in r.stderr + r.stdout
    assert not os.listdir(bin_dir / "render")
