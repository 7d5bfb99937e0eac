"""Renderer — the Python host's mirror of the reference's Renderer class
(include/renderer.hpp:32-52) on top of the C ABI.

    r = Renderer()                 # MAX_SCATTERINGS=4, SPP=4, SAMPLE_P=0.5
    r.SPP, r.MAX_SCATTERINGS, r.SAMPLE_P = 16, 8, 0.8
    buf = Rendering()
    r.render(scene, buf)           # Renderer::render, src/renderer.cpp:14
    tm = Rendering()
    r.toneMap(buf, tm, 0.12)       # Renderer::toneMap, src/renderer.cpp:149
    rgb8 = tm.rgb24()              # rendering::rgb24, include/renderer.hpp:20

Rendering runs on the GPU through liblambda_gpu.so; there is no CPU path.
"""
import ctypes

import numpy as np

from . import _lib as L
from .scene import FlatScene, SceneData


class Rendering:
    """rendering (include/renderer.hpp:16-30): img is (height, width, 3)
    linear RGB float32, row 0 at the top."""

    def __init__(self, img=None):
        self.img = img

    def rgb24(self, ctx=None):
        """8-bit sRGB of img (linRGB2sRGB then float2byte, cg.hpp:149-162)."""
        x = self.img.astype(np.float32)
        # the power only sees values of its own branch, so negative pixels
        # raise no warning; NaN maps to 0 as the device's encode does
        hi = np.power(np.maximum(x, np.float32(0.0031308)), np.float32(1 / 2.4))
        s = np.where(x > np.float32(0.0031308), np.float32(1.055) * hi - np.float32(0.055),
                     np.float32(12.92) * x)
        s = np.nan_to_num(s, nan=0.0, posinf=1.0, neginf=0.0)
        return np.clip((np.float32(255) * s + np.float32(0.5)).astype(np.int64), 0, 255).astype(np.uint8)


class Context:
    """One lgpu_ctx (one CUDA device, one uploaded scene)."""

    def __init__(self, device=0):
        self._lib = L.lib()
        h = ctypes.c_void_p()
        rc = self._lib.lgpu_create(int(device), ctypes.byref(h))
        L.check(None, rc, "lgpu_create")
        self.h = h
        self.flat = None
        self._scene_id = None

    def close(self):
        if self.h:
            self._lib.lgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, scene):
        flat = scene if isinstance(scene, FlatScene) else FlatScene(scene)
        L.check(self.h, self._lib.lgpu_upload_scene(self.h, flat.ptr()), "upload")
        self.flat = flat
        self._scene_id = id(scene)
        return flat

    def update_materials(self, flat):
        """Re-sends the materials and spectra of `flat` (same counts as the
        uploaded scene), e.g. after changing parameters in place."""
        L.check(self.h, self._lib.lgpu_update_materials(self.h, flat.ptr()), "update_materials")

    def upload_many(self, scenes):
        """Scene table for batched renders: scene k goes to slot k (slot 0
        is also the scene of render/trace)."""
        flats = [s if isinstance(s, FlatScene) else FlatScene(s) for s in scenes]
        arr = (ctypes.POINTER(L.Scene) * len(flats))(*[f.ptr() for f in flats])
        L.check(self.h, self._lib.lgpu_upload_scenes(self.h, arr, len(flats)), "upload_scenes")
        self.flat = flats[0]
        self.flats = flats
        self._scene_id = None
        return flats

    def slot_size(self, slot):
        c = self.flats[slot].scene.cam
        return int(c.width), int(c.height)

    @staticmethod
    def _jobs(jobs, outs):
        arr = (L.Job * len(jobs))()
        for k, (j, o) in enumerate(zip(jobs, outs)):
            arr[k].scene = int(j["scene"])
            arr[k].params = L.RenderParams(spp=int(j["spp"]), max_scatterings=int(j["max_scatterings"]),
                                           sample_p=float(j["sample_p"]), flags=int(j.get("flags", 0)),
                                           seed=int(j.get("seed", 0)),
                                           spp_offset=int(j.get("spp_offset", 0)))
            arr[k].out = o
            if "rect" in j:  # (x0, y0, width, height) from the top-left of the frame
                arr[k].x0, arr[k].y0, arr[k].width, arr[k].height = (int(v) for v in j["rect"])
        return arr

    def wave_config(self):
        c = L.WaveConfig()
        L.check(self.h, self._lib.lgpu_get_wave_config(self.h, ctypes.byref(c)), "get_wave_config")
        return {k: getattr(c, k) for k, _ in L.WaveConfig._fields_}

    def set_wave_config(self, **kw):
        """Changes fields of the wavefront launch shape (queue_cap,
        shade_block, trace_per_sm, graphs, mega_items)."""
        cur = self.wave_config()
        cur.update(kw)
        c = L.WaveConfig(**cur)
        L.check(self.h, self._lib.lgpu_set_wave_config(self.h, ctypes.byref(c)), "set_wave_config")

    def autotune_batch(self, jobs, spp_divisor=16):
        """Runs the library's autotuner on the jobs (spp / spp_divisor) and
        returns the launch shape it chose (now the context's)."""
        arr = self._jobs(jobs, [0] * len(jobs))
        c = L.WaveConfig()
        L.check(self.h, self._lib.lgpu_autotune_batch(self.h, arr, len(jobs), spp_divisor, ctypes.byref(c)),
                "autotune_batch")
        return {k: getattr(c, k) for k, _ in L.WaveConfig._fields_}

    def render_batch(self, jobs):
        """Renders every job (dicts: scene, spp, max_scatterings, sample_p
        and optionally seed, flags, spp_offset, rect = (x0, y0, width,
        height)) in one batched launch; returns one (height, width, 3) frame
        per job (a rect job fills only its rectangle; the rest is zero)."""
        imgs = []
        for j in jobs:
            s = int(j["scene"])
            # an unknown slot gets a placeholder; the library rejects the job
            w, h = self.slot_size(s) if 0 <= s < len(self.flats) else (1, 1)
            imgs.append(np.zeros((h, w, 3), np.float32))
        arr = self._jobs(jobs, [im.ctypes.data for im in imgs])
        L.check(self.h, self._lib.lgpu_render_batch(self.h, arr, len(jobs)), "render_batch")
        return imgs

    def render_batch_device(self, jobs, d_outs, stream=None):
        """render_batch with device outputs (pointers, one per job)."""
        arr = self._jobs(jobs, d_outs)
        L.check(self.h, self._lib.lgpu_render_batch_device(self.h, arr, len(jobs),
                                                           ctypes.c_void_p(stream or 0)),
                "render_batch_device")

    @property
    def size(self):
        c = self.flat.scene.cam
        return int(c.width), int(c.height)

    def render(self, spp, max_scatterings, sample_p, seed=0, flags=0, spp_offset=0, out=None):
        """The image (height, width, 3), row 0 at the top: float32, or
        float64 with flags containing FLAG_FP64_FILM."""
        w, h = self.size
        dt = np.float64 if flags & L.FLAG_FP64_FILM else np.float32
        if out is None:
            out = np.empty((h, w, 3), dt)
        assert out.dtype == dt and out.flags.c_contiguous and out.size == h * w * 3
        p = L.RenderParams(spp=spp, max_scatterings=max_scatterings, sample_p=sample_p, flags=flags,
                           seed=seed, spp_offset=spp_offset)
        L.check(self.h, self._lib.lgpu_render(self.h, ctypes.byref(p), out.ctypes.data), "render")
        return out

    def render_device(self, spp, max_scatterings, sample_p, d_out_ptr, seed=0, flags=0,
                      spp_offset=0, stream=None):
        p = L.RenderParams(spp=spp, max_scatterings=max_scatterings, sample_p=sample_p, flags=flags,
                           seed=seed, spp_offset=spp_offset)
        L.check(self.h, self._lib.lgpu_render_device(self.h, ctypes.byref(p), ctypes.c_void_p(d_out_ptr),
                                                     ctypes.c_void_p(stream or 0)), "render_device")

    def adjoint(self, spp, max_scatterings, sample_p, dloss_dimage, seed=0, flags=0, spp_offset=0,
                image=False):
        """Path-replay gradients of a loss whose image gradient is
        dloss_dimage ((height, width, 3), the render layout).  Returns
        (grad_spectra (n_spectra, n_bins), grad_materials (n_materials, 4):
        [thickness, alpha, 0, 0]) and, with image=True, the primal image of
        the same paths."""
        w, h = self.size
        sc = self.flat.scene
        d = np.ascontiguousarray(dloss_dimage, np.float32).reshape(h, w, 3)
        gs = np.zeros((int(sc.n_spectra), int(sc.spec.n_bins)), np.float32)
        gm = np.zeros((int(sc.n_materials), 4), np.float32)
        img = np.empty((h, w, 3), np.float32) if image else None
        p = L.RenderParams(spp=spp, max_scatterings=max_scatterings, sample_p=sample_p, flags=flags,
                           seed=seed, spp_offset=spp_offset)
        L.check(self.h, self._lib.lgpu_adjoint(self.h, ctypes.byref(p), d.ctypes.data, gs.ctypes.data,
                                               gm.ctypes.data, img.ctypes.data if image else None),
                "adjoint")
        return (gs, gm, img) if image else (gs, gm)

    def adjoint_device(self, spp, max_scatterings, sample_p, d_dimg, d_gspec, d_gmat, d_img=0, seed=0,
                       flags=0, spp_offset=0, stream=None):
        """adjoint() on device buffers (pointers)."""
        p = L.RenderParams(spp=spp, max_scatterings=max_scatterings, sample_p=sample_p, flags=flags,
                           seed=seed, spp_offset=spp_offset)
        L.check(self.h, self._lib.lgpu_adjoint_device(self.h, ctypes.byref(p), ctypes.c_void_p(d_dimg),
                                                      ctypes.c_void_p(d_gspec), ctypes.c_void_p(d_gmat),
                                                      ctypes.c_void_p(d_img or 0),
                                                      ctypes.c_void_p(stream or 0)), "adjoint_device")

    def trace(self, rays, flags=0):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = (L.Hit * max(rays.shape[0], 1))()
        L.check(self.h, self._lib.lgpu_trace_closest(self.h, rays.ctypes.data, rays.shape[0], flags,
                                                     ctypes.addressof(out)), "trace")
        return hits_to_numpy(out, rays.shape[0])

    def trace_any(self, rays, tmax, skip, flags=0):
        """Shadow-ray queries (lgpu_trace_any): for each ray, whether
        intersect::scene with the distance preset to tmax and object `skip`
        ignored (0xFFFFFFFF: none) finds a hit, i.e. the light is occluded."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        n = rays.shape[0]
        tmax = np.ascontiguousarray(np.broadcast_to(np.asarray(tmax, np.float32), (n,)))
        skip = np.ascontiguousarray(np.broadcast_to(np.asarray(skip, np.uint32), (n,)))
        out = np.zeros(max(n, 1), np.uint8)
        L.check(self.h, self._lib.lgpu_trace_any(self.h, rays.ctypes.data, tmax.ctypes.data, skip.ctypes.data,
                                                 n, flags, out.ctypes.data), "trace_any")
        return out[:n].astype(bool)

    def build_bvh(self, V, F, device=True):
        """bvh::build of a triangle mesh (V: positions (n, 3) with the
        loader's dummy at 0, F: (n_faces, k >= 3) vertex indices first) in
        the reference's layout, on this context's GPU (device=True) or with
        the host restatement.  Returns (nodes, bbs, prim_idxs)."""
        V = np.ascontiguousarray(V, np.float32).reshape(-1, 3)
        F = np.ascontiguousarray(F, np.uint32)
        nf, stride = F.shape
        nodes = np.zeros(4 * nf + 4, np.uint32)
        bbs = np.zeros(96 * nf + 96, np.float32)
        prims = np.zeros(nf + 1, np.uint32)
        nn, nb, npi = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        args = (V.ctypes.data, V.shape[0], F.ctypes.data, stride, nf, nodes.ctypes.data, ctypes.byref(nn),
                bbs.ctypes.data, ctypes.byref(nb), prims.ctypes.data, ctypes.byref(npi))
        if device:
            L.check(self.h, self._lib.lgpu_build_bvh_device(self.h, *args), "build_bvh_device")
        else:
            rc = self._lib.lgpu_build_bvh(*args)
            if rc != 0:
                raise L.LgpuError(rc, "lgpu_build_bvh failed")
        return nodes[:2 * nn.value].copy(), bbs[:48 * nb.value].copy(), prims[:npi.value].copy()

    def probe(self, queries):
        """Runs lgpu_probe_shading on a record array of _lib.PROBE_DTYPE;
        returns a record array of _lib.PROBE_RESULT_DTYPE."""
        q = np.ascontiguousarray(queries, L.PROBE_DTYPE)
        out = np.zeros(q.shape[0], L.PROBE_RESULT_DTYPE)
        L.check(self.h, self._lib.lgpu_probe_shading(self.h, q.ctypes.data, q.shape[0], out.ctypes.data),
                "probe")
        return out

    def tonemap(self, linrgb, y_mid=0.12):
        img = np.ascontiguousarray(linrgb, np.float32)
        h, w = img.shape[:2]
        tm = np.empty_like(img)
        b = np.empty(img.shape, np.uint8)
        L.check(self.h, self._lib.lgpu_tonemap(self.h, img.ctypes.data, w, h, y_mid, tm.ctypes.data,
                                               b.ctypes.data), "tonemap")
        return tm, b

    def stats(self):
        s = L.Stats()
        L.check(self.h, self._lib.lgpu_get_stats(self.h, ctypes.byref(s)), "stats")
        return {"last_kernel_ms": s.last_kernel_ms, "rays": s.rays, "paths": s.paths,
                "device_checks": s.device_checks, "max_stack": s.max_stack,
                "nonfinite_paths": s.nonfinite_paths, "node_tests": s.node_tests,
                "tri_tests": s.tri_tests, "inst_tests": s.inst_tests,
                "upload_bytes": s.upload_bytes, "launches": s.launches, "order_rays": s.order_rays,
                "local_stack": s.local_stack,
                "kernels": [{"ms": s.kernel_ms[k], "launches": s.kernel_launches[k],
                             "rays": s.kernel_rays[k], "node_tests": s.kernel_node_tests[k],
                             "tri_tests": s.kernel_tri_tests[k],
                             "inst_tests": s.kernel_inst_tests[k]} for k in range(3)]}


def hits_to_numpy(arr, n):
    """lgpu_hit array -> structured numpy array."""
    dt = np.dtype([("t", np.float32), ("obj", np.uint32), ("face", np.uint32), ("mat", np.uint32),
                   ("p", np.float32, 3), ("n", np.float32, 3), ("gn", np.float32, 3),
                   ("front", np.uint32)])
    assert dt.itemsize == ctypes.sizeof(L.Hit)
    buf = np.frombuffer(ctypes.string_at(ctypes.addressof(arr), n * dt.itemsize), dtype=dt)
    return buf.copy()


class Renderer:
    """Renderer (include/renderer.hpp:32-52).  render() uploads the scene
    when it is not the one uploaded last, then renders on the device."""

    def __init__(self, device=0, seed=0, flags=0):
        self.MAX_SCATTERINGS = 4
        self.SPP = 4
        self.SAMPLE_P = 0.5
        self.seed = seed
        self.flags = flags
        self.ctx = Context(device)

    def render(self, scene, buffer):
        if self.ctx._scene_id != id(scene):
            self.ctx.upload(scene)
        buffer.img = self.ctx.render(int(self.SPP), int(self.MAX_SCATTERINGS), float(self.SAMPLE_P),
                                     seed=self.seed, flags=self.flags)
        return buffer

    def toneMap(self, buffer, tm_buffer, Y_MID=0.12):
        tm, _ = self.ctx.tonemap(buffer.img, Y_MID)
        tm_buffer.img = tm
        return tm_buffer

    def tracePath(self, *args, **kwargs):
        raise NotImplementedError("single paths are traced inside the render kernel")
