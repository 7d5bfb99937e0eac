"""bench.py — throughput of lambda's spectral path-tracing render on B200.

Workload (the instanced configuration): 64 instances of one seeded displaced
icosphere (subdivision 7, 327,680 triangles) on a 2-triangle ground plane
under 2 quad lights; materials drawn uniformly from Lambertian / Blinn /
thin film; 1920x1080, 64 spp, 32 bounces, p = 0.8; the reference's spectral
constants (16 hero wavelengths on 400-720 nm, 80 bins).  Inputs are seeded
synthetic scenes (lambda_b200/synth.py) standing in for the reference's
benchmark scenes, which it does not ship.

A step is one render of the full frame: W*H*spp paths (one path = one
camera sample carrying 16 hero wavelengths, Renderer::tracePath).

    python bench.py [--gpus N --steps K --warmup W]       # device arm
    python bench.py --impl reference [...]                # reference CPU arm

value: Mpaths/s of the render kernel with the scene resident on the device
(CUDA events on the launching stream, L2 flushed between timed steps, max
over ranks).  e2e: the same metric through the C ABI with host buffers —
lgpu_upload_scene (host layout + host-to-device copies) plus lgpu_render
(kernel + device-to-host image) per step.  Multi-GPU: every rank renders
its own frame (weak scaling, no collective on the data path).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = ("Mpaths/s at fixed RMSE: plain GPU vs batched vs host CPU; adjoint/forward cost")
UNIT = "Mpaths/s"

FULL = dict(n_instances=64, subdiv=7, width=1920, spp=64, bounces=32, p=0.8)
SMALL = dict(n_instances=64, subdiv=7, width=480, spp=2, bounces=32, p=0.8)

# per-unit algorithmic bytes of the traversal (one 8-wide node: 6x8 float
# bounds + 8 B header; one triangle: 3 float3 vertices; one instance test:
# M and M_inv; one hit: shading normals + material header)
BYTES_PER_NODE = 200
BYTES_PER_TRI = 36
BYTES_PER_INST = 128
BYTES_PER_RAY = 64


def workload_desc(w):
    return ("instanced: %d x displaced icosphere (subdivision %d, %d tris), 2-tri ground, "
            "2 quad lights, %dx%d, %d spp, %d bounces, p=%.1f, 16 hero wavelengths 400-720 nm "
            "(80 bins)" % (w["n_instances"], w["subdiv"], 20 * 4 ** w["subdiv"], w["width"],
                           int(round(w["width"] * 9 / 16)), w["spp"], w["bounces"], w["p"]))


def make_scene(w, cache=None):
    from lambda_b200 import synth
    cache = cache or os.environ.get("LGPU_BENCH_CACHE") or os.path.join(tempfile.gettempdir(),
                                                                       "lgpu_bench")
    d = os.path.join(cache, "instanced_%d_%d_%d" % (w["n_instances"], w["subdiv"], w["width"]))
    nls = os.path.join(d, "scene.nls")
    if not os.path.exists(nls):
        synth.instanced(d, n_instances=w["n_instances"], subdiv=w["subdiv"], width=w["width"])
    return nls


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic_per_ray(kind):
    """DRAM bytes (read + write) per ray of kernel kind (0 closest-hit,
    1 shadow) from the committed ncu summary
    profiles/traffic_instanced.json, or None."""
    p = os.path.join(REPO, "profiles", "traffic_instanced.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["dram_bytes_per_ray"][str(kind)])
    except (OSError, KeyError, ValueError, TypeError):
        return None


KERNEL_NAMES = ("closest-hit traversal (wf_trace_persistent<false> + wf_trace_fallback)",
                "shadow traversal (wf_trace_persistent<true>)", "shading (wf_shade)")


def kernel_roofline(ctx, spp, B, p, stream):
    """Roofline of the dominant kernel from one untimed render with
    per-kernel timing (CUDA events around every traversal and shading
    launch on the render stream, separate work counters per kind).
    achieved = algorithmic bytes of its launches / their summed device
    time; the algorithmic bytes are its node, triangle, instance and ray
    counts times BYTES_PER_*."""
    import torch

    from lambda_b200 import _lib as L
    W, H = ctx.size
    d_out = torch.empty(W * H * 3, dtype=torch.float32, device="cuda")
    ctx.render_device(spp, B, p, d_out.data_ptr(), seed=77, flags=L.FLAG_KERNEL_TIMING,
                      stream=stream.cuda_stream)
    torch.cuda.synchronize()
    ks = ctx.stats()["kernels"]
    top = max(range(3), key=lambda k: ks[k]["ms"])
    k = ks[top]
    total_ms = sum(x["ms"] for x in ks)
    peak, peak_kind = measured_peak_hbm()
    if top == 2 or k["ms"] <= 0:
        algo = None
        achieved = None
    else:
        algo = (k["node_tests"] * BYTES_PER_NODE + k["tri_tests"] * BYTES_PER_TRI +
                k["inst_tests"] * BYTES_PER_INST + k["rays"] * BYTES_PER_RAY)
        achieved = algo / (k["ms"] / 1e3) / 1e9
    launches = max(int(k["launches"]), 1)
    tpr = profile_traffic_per_ray(top)
    tpl = tpr * k["rays"] / launches if tpr is not None else None
    return {"bound": "hbm", "kernel": KERNEL_NAMES[top], "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": (achieved / peak) if achieved is not None else None,
            "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
            else peak_kind,
            "traffic": tpl,
            "algorithmic_bytes_per_launch": (algo / launches) if algo is not None else None,
            "avg_launch_ms": k["ms"] / launches, "launches": int(k["launches"]),
            "share_of_kernel_time": k["ms"] / total_ms if total_ms > 0 else None,
            "per_launch": {"rays": k["rays"] / launches, "node_tests": k["node_tests"] / launches,
                           "tri_tests": k["tri_tests"] / launches,
                           "inst_tests": k["inst_tests"] / launches},
            "mrays_per_s": k["rays"] / (k["ms"] / 1e3) / 1e6 if k["ms"] > 0 else None,
            "kernels_ms": {KERNEL_NAMES[i].split(" (")[0]: ks[i]["ms"] for i in range(3)}}


BATCH_DESC = ("64 jobs: box room (10 wall tris + 2 blocks, quad light) with U[1,128] instances of a "
              "displaced icosphere of subdivision 5-7 (20K-328K tris each), resolution from "
              "128^2/256^2/512^2/1024^2, spp log-uniform 4-256, bounces U[4,32], p=0.8, "
              "4 hero wavelengths on 380-780 nm (81 bins)")


def run_batched(ctx_cls, device, n_jobs=64):
    """Config 3: the 64 jobs in one batched launch vs the same jobs as
    back-to-back plain launches (lgpu_render_batch_device with one job),
    scenes resident, device time by CUDA events; both produce identical
    images (checked), so per-job RMSE is equal."""
    import numpy as np
    import torch

    from lambda_b200 import synth
    from lambda_b200.scene import SpectralConfig, flatten, load_nls
    root = os.path.join(tempfile.gettempdir(), "lgpu_bench", "batch")
    cfg = SpectralConfig(n_bins=81, lambda_inf=380.0, lambda_sup=780.0, hero_k=4)
    specs = synth.batch_jobs(n_jobs)
    flats = []
    for k, j in enumerate(specs):
        nls = synth.batch_job(os.path.join(root, "job%02d" % k), j["n_instances"], j["subdiv"],
                              os.path.join(root, "meshes"), seed=j["seed"], width=j["width"])
        flats.append(flatten(load_nls(nls, cfg)))
    ctx = ctx_cls(device)
    ctx.upload_many(flats)
    jobs = [dict(scene=k, spp=j["spp"], max_scatterings=j["max_scatterings"], sample_p=j["sample_p"],
                 seed=j["seed"]) for k, j in enumerate(specs)]
    outs = [torch.empty(j["width"] * j["width"] * 3, dtype=torch.float32, device="cuda") for j in specs]
    seq = [torch.empty_like(o) for o in outs]
    ptrs = [o.data_ptr() for o in outs]
    paths = sum(j["width"] * j["width"] * j["spp"] for j in specs)
    stream = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def timed(fn):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    def batched():
        ctx.render_batch_device(jobs, ptrs, stream=stream.cuda_stream)

    def sequential():
        for j, o in zip(jobs, seq):
            ctx.render_batch_device([j], [o.data_ptr()], stream=stream.cuda_stream)

    batched()
    launches = ctx.stats()["launches"]
    sequential()
    t_b = timed(batched)
    t_s = timed(sequential)
    equal = all(torch.equal(a, b) for a, b in zip(outs, seq))
    # the library's autotuner on the same jobs at spp / 16, then the batch
    # again with the launch shape it chose
    t0 = time.perf_counter()
    cfg = ctx.autotune_batch(jobs, spp_divisor=16)
    tune_s = time.perf_counter() - t0
    batched()
    t_t = timed(batched)
    equal_t = all(torch.equal(a, b) for a, b in zip(outs, seq)) if not cfg["mega_items"] else None
    return {"value": paths / t_t / 1e6, "unit": UNIT, "sequential_value": paths / t_s / 1e6,
            "speedup": t_s / t_t, "batched_default_value": paths / t_b / 1e6,
            "speedup_default_config": t_s / t_b, "batched_s": t_t, "batched_default_s": t_b,
            "sequential_s": t_s, "paths": paths, "jobs": n_jobs, "images_identical": bool(equal),
            "images_identical_tuned": equal_t, "autotune": {"config": cfg, "seconds": tune_s},
            "gpu_launches": int(launches), "workload": BATCH_DESC}


ADJ_DESC = ("inverse-rendering scene: 64x64 thin-film tiles (one object and material each) under 64 "
            "Lambertian UV spheres (48K tris), 2 quad lights; 512x512, 32 spp, 4 bounces, p=0.8, "
            "16 hero wavelengths 400-720 nm (80 bins); parameters 64x32 albedo samples + 64x64 thickness")


def run_adjoint(device, n_fd=100, reps=3):
    """Config 4: forward render vs path-replay adjoint (device time, CUDA
    events), and the adjoint against central finite differences of the
    device renderer with common random numbers on n_fd random parameters
    (loss <w, image> with a fixed seeded weight image w)."""
    import numpy as np
    import torch

    from lambda_b200 import synth
    from lambda_b200.inverse import DiffScene
    rng = np.random.default_rng(4)
    alb = rng.uniform(0.1, 0.9, (64, synth.ALBEDO_BINS))
    th = rng.uniform(200.0, 800.0, (64, 64))
    sc = DiffScene(alb, th, width=512, spp=32, bounces=4, device=device)
    sc.set_params(alb, th)
    ctx = sc.ctx
    H, W, _ = sc.shape
    wimg = np.random.default_rng(5).standard_normal((H, W, 3)).astype(np.float32)
    d_w = torch.from_numpy(wimg).cuda()
    d_img = torch.empty(H * W * 3, dtype=torch.float32, device="cuda")
    n_spec = int(sc.flat.scene.n_spectra) * int(sc.flat.scene.spec.n_bins)
    d_gs = torch.empty(n_spec, dtype=torch.float32, device="cuda")
    d_gm = torch.empty(4 * int(sc.flat.scene.n_materials), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    def fwd():
        ctx.render_device(sc.spp, sc.bounces, sc.p, d_img.data_ptr(), seed=7, stream=stream.cuda_stream)

    def adj():
        ctx.adjoint_device(sc.spp, sc.bounces, sc.p, d_w.data_ptr(), d_gs.data_ptr(), d_gm.data_ptr(), seed=7,
                           stream=stream.cuda_stream)

    fwd()
    adj()
    t_f = min(timed(fwd) for _ in range(reps))
    t_a = min(timed(adj) for _ in range(reps))
    g_alb, g_th = sc.gradients(wimg, seed=7)
    paths = H * W * sc.spp

    def loss():
        return float(np.sum(sc.render(seed=7).astype(np.float64) * wimg))

    def fd_check(h_alb, h_th_rel):
        """central differences with the given steps on n_fd random parameters"""
        frng = np.random.default_rng(11)
        live_a = np.argwhere(g_alb != 0)
        live_t = np.argwhere(g_th != 0)
        out = []
        for k in range(n_fd):
            if frng.uniform() < 0.5 or len(live_t) == 0:
                i, j = (int(x) for x in live_a[frng.integers(len(live_a))])
                h, g = h_alb, g_alb[i, j]
                a = alb.copy()
                a[i, j] += h
                sc.set_params(a, th)
                lp = loss()
                a[i, j] -= 2 * h
                sc.set_params(a, th)
                lm = loss()
                name = "albedo"
            else:
                i, j = (int(x) for x in live_t[frng.integers(len(live_t))])
                h, g = h_th_rel * th[i, j], g_th[i, j]
                t = th.copy()
                t[i, j] += h
                sc.set_params(alb, t)
                lp = loss()
                t[i, j] -= 2 * h
                sc.set_params(alb, t)
                lm = loss()
                name = "thickness"
            out.append((name, i, j, float(g), (lp - lm) / (2 * h)))
        sc.set_params(alb, th)
        g = np.array([[o[3], o[4]] for o in out])
        rel = np.abs(g[:, 0] - g[:, 1]) / np.maximum(np.abs(g[:, 1]), 1e-30)
        worst = np.argsort(-rel)[:3]
        return {"h": "%g (albedo) / %g x thickness" % (h_alb, h_th_rel),
                "rel_err_median": float(np.median(rel)), "rel_err_max": float(rel.max()),
                "within_2pct": int(np.sum(rel <= 0.02)), "worst": [list(out[w]) for w in worst],
                "drawn_from": "%d albedo samples, %d tiles with a non-zero adjoint gradient" %
                              (len(live_a), len(live_t))}

    fd3 = fd_check(1e-3, 1e-3)
    fd2 = fd_check(1e-2, 1e-2)
    return {"forward_s": t_f, "adjoint_s": t_a, "cost_ratio": t_a / t_f,
            "forward_mpaths_s": paths / t_f / 1e6, "fd_params": n_fd,
            "fd": "central differences of the device renderer, same seed (common random numbers), loss "
                  "<w, image> with a seeded normal weight image; relative error |adjoint - fd| / |fd|",
            "fd_h1e-3": fd3, "fd_h1e-2": fd2, "workload": ADJ_DESC}


LARGE = dict(n_instances=256, width=3840, spp=256, bounces=32, p=0.8)
LARGE_DESC = ("large: 256 instances of a 65,536-triangle displaced UV sphere (16.8M instanced tris), 2-tri "
              "ground, 2 quad lights, 3840x2160, 256 spp, 32 bounces, p=0.8, 16 hero wavelengths 400-720 nm "
              "(80 bins); 16 tile jobs (4x4) of the frame in one batched launch; one adjoint pass (all "
              "albedo and thin-film IOR spectra, thicknesses, exponents)")


def run_large(args):
    """Config 5: the 4K frame as 16 tile jobs in one batched launch, the
    same frame as one plain render, and one adjoint pass of it."""
    import numpy as np
    import torch

    from lambda_b200 import synth
    from lambda_b200.renderer import Context
    from lambda_b200.scene import flatten, load_nls
    w = dict(LARGE)
    if args.spp:
        w["spp"] = args.spp
    root = os.path.join(tempfile.gettempdir(), "lgpu_bench", "large")
    nls = synth.instanced(root, n_instances=w["n_instances"], width=w["width"], mesh="uv64k")
    fs = flatten(load_nls(nls))
    ctx = Context(0)
    ctx.upload_many([fs])
    W, H = ctx.size
    paths = W * H * w["spp"]
    d_out = torch.zeros(W * H * 3, dtype=torch.float32, device="cuda")
    d_tiles = torch.zeros_like(d_out)
    stream = torch.cuda.current_stream()
    job = dict(scene=0, spp=w["spp"], max_scatterings=w["bounces"], sample_p=w["p"], seed=3)
    xs = [W * k // 4 for k in range(5)]
    ys = [H * k // 4 for k in range(5)]
    tiles = [dict(job, rect=(xs[a], ys[b], xs[a + 1] - xs[a], ys[b + 1] - ys[b])) for b in range(4)
             for a in range(4)]

    def timed(fn):
        # the second of two runs: the first also sizes the context's buffers
        # for the call (tens of GB at this size)
        for _ in range(2):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    t_plain = timed(lambda: ctx.render_device(w["spp"], w["bounces"], w["p"], d_out.data_ptr(), seed=3,
                                              stream=stream.cuda_stream))
    t_tiles = timed(lambda: ctx.render_batch_device(tiles, [d_tiles.data_ptr()] * 16, stream=stream.cuda_stream))
    same = bool(torch.equal(d_out, d_tiles))
    wimg = torch.from_numpy(np.random.default_rng(5).standard_normal(H * W * 3).astype(np.float32)).cuda()
    n_spec = int(fs.scene.n_spectra) * int(fs.scene.spec.n_bins)
    d_gs = torch.zeros(n_spec, dtype=torch.float32, device="cuda")
    d_gm = torch.zeros(4 * int(fs.scene.n_materials), dtype=torch.float32, device="cuda")
    t_adj = timed(lambda: ctx.adjoint_device(w["spp"], w["bounces"], w["p"], wimg.data_ptr(), d_gs.data_ptr(),
                                             d_gm.data_ptr(), seed=3, stream=stream.cuda_stream))
    line = {"metric": METRIC, "value": paths / t_tiles / 1e6, "unit": UNIT, "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": t_tiles * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": {"workload": LARGE_DESC, "paths": paths},
            "plain_value": paths / t_plain / 1e6, "tiles_identical_to_plain": same,
            "adjoint_s": t_adj, "adjoint_cost_ratio": t_adj / t_plain,
            "gradient_nonzero": int((d_gs != 0).sum().item() + (d_gm != 0).sum().item())}
    print(json.dumps(line))
    return 0


def rmse_check(ctx, w, ref_rows, d_out, stream, oracle_renders=16):
    """Relative RMSE per channel, over the reference's sampled rows, of the
    device image and of the reference's own image at the workload's spp,
    both against an FP64 mean of oracle_renders device renders of that spp
    with other random streams (the high-spp oracle image)."""
    import numpy as np
    import torch
    W, H = ctx.size
    spp, B, p = w["spp"], w["bounces"], w["p"]
    acc = np.zeros((H, W, 3), np.float64)
    for k in range(oracle_renders):
        ctx.render_device(spp, B, p, d_out.data_ptr(), seed=999, spp_offset=k * spp,
                          stream=stream.cuda_stream)
        torch.cuda.synchronize()
        acc += d_out.cpu().numpy().reshape(H, W, 3)
    oracle = acc / oracle_renders
    ctx.render_device(spp, B, p, d_out.data_ptr(), seed=1, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    gpu = d_out.cpu().numpy().reshape(H, W, 3).astype(np.float64)
    rows = sorted(ref_rows)
    # scene row r is image row H - 1 - r
    o = np.stack([oracle[H - 1 - r] for r in rows])
    g = np.stack([gpu[H - 1 - r] for r in rows])
    c = np.stack([ref_rows[r].astype(np.float64) for r in rows])
    den = np.sqrt(np.mean(o ** 2, axis=(0, 1)))
    e_g = np.sqrt(np.mean((g - o) ** 2, axis=(0, 1))) / den
    e_c = np.sqrt(np.mean((c - o) ** 2, axis=(0, 1))) / den
    # means over the rows: a bias between the estimators would show here
    mean_ratio = np.mean(c, axis=(0, 1)) / np.mean(o, axis=(0, 1))
    return {"device": [float(x) for x in e_g], "reference": [float(x) for x in e_c],
            "ratio": [float(x) for x in e_g / e_c], "rows": len(rows),
            "reference_mean_over_oracle_mean": [float(x) for x in mean_ratio],
            "oracle": "device, %d spp (%d renders of %d spp with other random streams, FP64 mean)" %
                      (oracle_renders * spp, oracle_renders, spp),
            "what": "relative RMSE per channel (R, G, B) over the reference's sampled rows at %d spp" % spp}


def cpu_reference_sample(nls, w, budget_s, fast=True, keep=None):
    """Times the reference's own pixel loop (oracle/_ref, -O3 OpenMP build)
    over rows spread across the image; returns (paths/s, cores, sample).
    With a dict `keep`, the rendered rows are stored in it by scene row."""
    from oracle import refharness
    ref = refharness.RefScene(nls, fast=fast)
    cores = ref.L.ref_max_threads()
    H = ref.height
    t0 = time.perf_counter()
    ref.render_rows(w["spp"], w["bounces"], w["p"], H // 2, H // 2 + 1)
    one = max(time.perf_counter() - t0, 1e-3)
    n_rows = int(max(1, min(H, budget_s / one)))
    rows = sorted(set(int(round(x)) for x in
                      [i * (H - 1) / max(n_rows - 1, 1) for i in range(n_rows)]))
    t0 = time.perf_counter()
    for r in rows:
        img = ref.render_rows(w["spp"], w["bounces"], w["p"], r, r + 1)
        if keep is not None:
            keep[r] = img[0]
    dt = time.perf_counter() - t0
    paths = len(rows) * ref.width * w["spp"]
    sample = "%d of %d rows (evenly spread) x %d px x %d spp = %d paths" % (
        len(rows), H, ref.width, w["spp"], paths)
    return paths / dt, cores, sample


def run_reference(args, w):
    rank = rank_env()[1]
    if rank != 0:
        return 0
    from oracle import refharness
    if not refharness.available(fast=True):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libref_fast.so was not built"}))
        return 0
    nls = make_scene(w)
    for _ in range(args.warmup):
        cpu_reference_sample(nls, w, args.ref_step_s)
    vals, cores, sample = [], 0, ""
    for _ in range(args.steps):
        v, cores, sample = cpu_reference_sample(nls, w, args.ref_step_s)
        vals.append(v)
    value = statistics.mean(vals) / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": workload_desc(w), "cpu": "reference Renderer pixel loop, "
                       "-O3 -fopenmp -march=x86-64-v3 build of the reference sources"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def rank_env():
    """(world size, rank, local rank) as torch.distributed.run sets them."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(x, dist, device):
    """The largest x over all ranks (x itself without a process group)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(paths_per_step, steps, world, total_ms):
    """Whole-job Mpaths/s: every rank renders its own frame of paths_per_step
    paths each step (replicas, weak scaling), and the job takes as long as
    its slowest rank (total_ms, the max over ranks)."""
    return world * paths_per_step * steps / (total_ms / 1e3) / 1e6


def run_device(args, w):
    import torch

    from lambda_b200.renderer import Context
    from lambda_b200.scene import flatten, load_nls

    world, rank, local = rank_env()
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)

    nls = make_scene(w)
    sc = load_nls(nls)
    fs = flatten(sc)
    ctx = Context(local)
    ctx.upload(fs)
    if args.queue_cap:
        ctx.set_wave_config(queue_cap=args.queue_cap)
    W, H = ctx.size
    spp, B, p = w["spp"], w["bounces"], w["p"]
    paths_per_step = W * H * spp
    d_out = torch.empty(W * H * 3, dtype=torch.float32, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    stream = torch.cuda.current_stream()

    def step(seed):
        ctx.render_device(spp, B, p, d_out.data_ptr(), seed=seed, stream=stream.cuda_stream)

    for k in range(args.warmup):
        step(1000 + k)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    step_ms, kern_ms, counters = [], [], []
    for k in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step(k)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        st = ctx.stats()
        kern_ms.append(st["last_kernel_ms"])
        counters.append(st)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(step_ms), dist, "cuda")
    value = job_throughput(paths_per_step, args.steps, world, total_ms)

    # end to end through the C ABI with host buffers
    import numpy as np
    host = np.empty((H, W, 3), np.float32)
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        ctx.upload(fs)
        ctx.render(spp, B, p, seed=k, out=host)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
    h2d = ctx.stats()["upload_bytes"]
    e2e = {"value": job_throughput(paths_per_step, e2e_steps, world, e2e_s * 1e3), "unit": UNIT,
           "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(W * H * 3 * 4),
           "note": "lgpu_upload_scene (host layout + copies) + lgpu_render (kernel + image "
                   "readback) per step"}

    c = counters[-1]
    launches_per_step = int(c["launches"])
    roofline = kernel_roofline(ctx, spp, B, p, stream)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generator)",
            "config": {"workload": workload_desc(w), "paths_per_step_per_gpu": paths_per_step,
                       "l2": "256 MB buffer written between timed steps",
                       "parallelism": "frame per GPU" if world > 1 else "single GPU"},
            "e2e": e2e, "roofline": roofline, "clocks": clk,
            "gpu_launches": launches_per_step * args.steps,
            "mrays_per_s": world * c["rays"] * args.steps / (total_ms / 1e3) / 1e6}
    if rank == 0 and world == 1 and not args.no_batch:
        line["batched"] = run_batched(Context, local)
    if rank == 0 and world == 1 and not args.no_adjoint:
        line["adjoint"] = run_adjoint(local)
    if rank == 0 and world == 1 and not args.no_baseline:
        from oracle import refharness
        if refharness.available(fast=True):
            rows = {}
            v, cores, sample = cpu_reference_sample(nls, w, args.ref_step_s, keep=rows)
            line["cpu_baseline"] = {"value": v / 1e6, "unit": UNIT, "cores": cores,
                                    "kind": "reference", "sample": sample}
            line["rmse"] = rmse_check(ctx, w, rows, d_out, stream)
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="lgpu", choices=["lgpu", "reference"])
    ap.add_argument("--small", action="store_true", help="reduced frame (profiling)")
    ap.add_argument("--spp", type=int, default=None)
    ap.add_argument("--width", type=int, default=None, help="frame width (profiling)")
    ap.add_argument("--queue-cap", type=int, default=0,
                    help="paths in flight (profiling a launch of a given size; default: the library's)")
    ap.add_argument("--no-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-vs-sequential run")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint cost and FD check")
    ap.add_argument("--large", action="store_true",
                    help="the large configuration (4K, 16 tile jobs, one adjoint pass) instead")
    ap.add_argument("--ref-step-s", type=float, default=8.0,
                    help="seconds of reference CPU work per sampled step")
    args = ap.parse_args()
    w = dict(SMALL if args.small else FULL)
    if args.spp:
        w["spp"] = args.spp
    if args.width:
        w["width"] = args.width
    if args.impl == "reference":
        return run_reference(args, w)
    if args.large:
        return run_large(args)
    return run_device(args, w)


if __name__ == "__main__":
    sys.exit(main())
