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

Beside the headline (N=1, rank 0): roofline (HBM, FP32 and issue bounds of
the dominant kernel), cpu_baseline (the reference's own pixel loop on the
host's cores), rmse (fixed-RMSE check against the reference's FP64 film),
batched (config 3: 64 jobs in one launch vs back to back), adjoint (config
4: cost and finite-difference check), box_room (config 1, against the
reference built at 4 hero wavelengths, 81 bins on 380-780 nm) and large
(config 5: a 4K frame as 16 tile jobs, one adjoint pass).
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
# per-unit FP32 operations of the traversal, counted from the kernel source
# (lgpu_intersect.cuh; every operation is one instruction, the library is
# built without multiply-add contraction): an 8-wide node test is 8 children
# x (6 subtractions + 6 multiplications + 3 max + 3 min + 1 compare) plus 28
# compares ranking the hit children; a full triangle test (tri_test) 108; an
# instance entry (two 3x4 transforms, the inverse direction, the mesh-bounds
# slab test, the ray's moment) 80
FLOPS_PER_NODE = 8 * 19 + 28
FLOPS_PER_TRI = 108
FLOPS_PER_INST = 80
# B200: 148 SMs, 128 FP32 lanes and 4 warp schedulers (one instruction per
# cycle each) per SM
N_SM, FP32_LANES, SCHEDULERS = 148, 128, 4


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


def profile_per_ray(kind, key="dram_bytes_per_ray"):
    """A per-ray figure of kernel kind (0 closest-hit, 1 shadow) from the
    committed ncu summary profiles/traffic_instanced.json: DRAM bytes (read
    + write) or warp instructions issued, per traced ray; None if absent."""
    p = os.path.join(REPO, "profiles", "traffic_instanced.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d[key][str(kind)])
    except (OSError, KeyError, ValueError, TypeError):
        return None


KERNEL_NAMES = ("closest-hit traversal (wf_trace_persistent<false> + wf_trace_fallback)",
                "shadow traversal (wf_trace_persistent<true>)", "shading (wf_shade)")


def kernel_roofline(ctx, spp, B, p, stream, sm_mhz=None):
    """Roofline of the dominant kernel from one untimed render with
    per-kernel timing (CUDA events around every traversal and shading
    launch on the render stream, separate work counters per kind), against
    three bounds:
      hbm    algorithmic bytes (node, triangle, instance and ray counts x
             BYTES_PER_*) / its summed device time, against the measured
             copy bandwidth (MEASURED_PEAKS.json);
      fp32   algorithmic FP32 operations (FLOPS_PER_*) / time, against 148
             SMs x 128 lanes x the SM clock sampled during the run;
      issue  warp instructions issued (per ray, from the committed ncu
             summary, x the rays) / time, against 148 SMs x 4 schedulers x
             the SM clock.
    `bound` names the largest fraction; achieved/peak/unit/frac are that
    bound's, and every bound's figures are listed under `bounds`."""
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
    tpr = profile_per_ray(top)
    tpl = tpr * k["rays"] / launches if tpr is not None else None
    mhz = float(sm_mhz or 1965.0)
    secs = k["ms"] / 1e3
    bounds = {"hbm": {"achieved": achieved, "peak": peak, "unit": "GB/s",
                      "frac": (achieved / peak) if achieved is not None else None,
                      "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                      else peak_kind + " (6650 GB/s)"}}
    if top != 2 and secs > 0:
        ops = (k["node_tests"] * FLOPS_PER_NODE + k["tri_tests"] * FLOPS_PER_TRI +
               k["inst_tests"] * FLOPS_PER_INST)
        pk = N_SM * FP32_LANES * mhz * 1e6 / 1e12
        bounds["fp32"] = {"achieved": ops / secs / 1e12, "peak": pk, "unit": "TFLOP/s",
                          "frac": ops / secs / 1e12 / pk,
                          "peak_source": "148 SMs x 128 FP32 lanes x %.0f MHz (SM clock sampled during the run); "
                                         "no multiply-add contraction, one operation per instruction" % mhz}
        ipr = profile_per_ray(top, "warp_inst_per_ray")
        if ipr is not None:
            inst = ipr * k["rays"]
            pk = N_SM * SCHEDULERS * mhz * 1e6 / 1e12
            bounds["issue"] = {"achieved": inst / secs / 1e12, "peak": pk, "unit": "Twarp-inst/s",
                               "frac": inst / secs / 1e12 / pk, "warp_inst_per_ray": ipr,
                               "peak_source": "148 SMs x 4 schedulers x %.0f MHz; instructions per ray from "
                                              "profiles/traffic_instanced.json (ncu smsp__inst_executed.sum)"
                                              % mhz}
    binding = max((b for b in bounds if bounds[b]["frac"] is not None), key=lambda b: bounds[b]["frac"],
                  default="hbm")
    bb = bounds[binding]
    return {"bound": binding, "kernel": KERNEL_NAMES[top], "achieved": bb["achieved"], "peak": bb["peak"],
            "unit": bb["unit"], "frac": bb["frac"], "peak_source": bb["peak_source"], "bounds": bounds,
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
    # each job alone, timed: the best rate any job reaches alone is the
    # steady state of the wavefront on these scenes; batching can at best
    # run every path at that rate, so total paths / that rate bounds the
    # batched time from below and t_s / it the speedup from above
    job_paths = [j["width"] * j["width"] * j["spp"] for j in specs]
    job_s = [timed(lambda j=j, o=o: ctx.render_batch_device([j], [o.data_ptr()], stream=stream.cuda_stream))
             for j, o in zip(jobs, seq)]
    best_rate = max(pth / t for pth, t in zip(job_paths, job_s))
    bound = t_s / (paths / best_rate)
    # the small jobs (at most 256x256 pixels and 16 spp): batched vs back to back
    small = [k for k, j in enumerate(specs) if j["width"] <= 256 and j["spp"] <= 16]
    small_paths = sum(job_paths[k] for k in small)
    t_bs = timed(lambda: ctx.render_batch_device([jobs[k] for k in small], [ptrs[k] for k in small],
                                                 stream=stream.cuda_stream)) if small else 0.0
    t_ss = timed(lambda: [ctx.render_batch_device([jobs[k]], [seq[k].data_ptr()], stream=stream.cuda_stream)
                          for k in small]) if small else 0.0
    # the library's autotuner on the same jobs at spp / 16, then the batch
    # again with the launch shape it chose
    t0 = time.perf_counter()
    cfg = ctx.autotune_batch(jobs, spp_divisor=16)
    tune_s = time.perf_counter() - t0
    batched()
    t_t = timed(batched)
    equal_t = all(torch.equal(a, b) for a, b in zip(outs, seq)) if not cfg["mega_items"] else None
    return {"value": paths / t_t / 1e6, "unit": UNIT, "sequential_value": paths / t_s / 1e6,
            "speedup": t_s / t_t, "speedup_bound": bound,
            "bound": "sequential time / (total paths / the best rate of any job rendered alone, %.1f Mpaths/s): "
                     "what batching could gain if every path ran at the steady-state rate" % (best_rate / 1e6),
            "small_jobs": {"jobs": len(small), "paths": small_paths,
                           "batched_value": small_paths / t_bs / 1e6 if t_bs else None,
                           "sequential_value": small_paths / t_ss / 1e6 if t_ss else None,
                           "speedup": t_ss / t_bs if t_bs else None,
                           "what": "the jobs of at most 256x256 pixels and 16 spp, batched vs back to back"},
            "batched_default_value": paths / t_b / 1e6,
            "speedup_default_config": t_s / t_b, "batched_s": t_t, "batched_default_s": t_b,
            "sequential_s": t_s, "paths": paths, "jobs": n_jobs, "images_identical": bool(equal),
            "images_identical_tuned": equal_t, "autotune": {"config": cfg, "seconds": tune_s},
            "gpu_launches": int(launches), "workload": BATCH_DESC}


ADJ_DESC = ("inverse-rendering scene: 64x64 thin-film tiles (one object and material each) under 64 "
            "Lambertian UV spheres (48K tris), 2 quad lights; 512x512, 32 spp, 4 bounces, p=0.8, "
            "16 hero wavelengths 400-720 nm (80 bins); parameters 64x32 albedo samples + 64x64 thickness; "
            "L2 loss against a 1024-spp target rendered with hidden parameters")
FD_H = 1e-3          # albedo samples: absolute; thickness: relative
FD_FLOOR = 0.01      # relative errors are taken against max(|fd|, FD_FLOOR x RMS of the checked fds)


def run_adjoint(device, n_fd=100, reps=3):
    """Config 4: the forward render vs the path-replay adjoint (device time,
    CUDA events), and the adjoint against central finite differences of
    the device renderer with common random numbers on n_fd random
    parameters.  Loss = sum((I - T)^2) against a target T rendered at 1024
    spp with hidden parameters (thickness U[200, 800] nm, albedo random);
    the parameters sit at the initial guess (thickness 400 nm, albedo 0.5).
    Finite differences render with the FP64 film (LGPU_FLAG_FP64_FILM) at
    h = FD_H, so the float film's rounding does not swamp them."""
    import numpy as np
    import torch

    from lambda_b200 import _lib as L
    from lambda_b200 import synth
    from lambda_b200.inverse import DiffScene
    rng = np.random.default_rng(4)
    alb_true = np.clip(rng.uniform(0.1, 0.9, (64, 1)) + 0.1 * rng.standard_normal((64, synth.ALBEDO_BINS)),
                       0.05, 0.95)
    th_true = rng.uniform(200.0, 800.0, (64, 64))
    alb = np.full((64, synth.ALBEDO_BINS), 0.5)
    th = np.full((64, 64), 400.0)
    sc = DiffScene(alb, th, width=512, spp=32, bounces=4, device=device)
    sc.set_params(alb_true, th_true)
    target = sc.ctx.render(1024, sc.bounces, sc.p, seed=99, flags=L.FLAG_FP64_FILM)
    sc.set_params(alb, th)
    ctx = sc.ctx
    H, W, _ = sc.shape
    seed = 7

    def img_fp64():
        return ctx.render(sc.spp, sc.bounces, sc.p, seed=seed, flags=L.FLAG_FP64_FILM)

    def loss():
        return float(np.sum((img_fp64() - target) ** 2))

    dimg = (2.0 * (img_fp64() - target)).astype(np.float32)
    d_w = torch.from_numpy(dimg).cuda()
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
        ctx.render_device(sc.spp, sc.bounces, sc.p, d_img.data_ptr(), seed=seed, stream=stream.cuda_stream)

    def adj():
        ctx.adjoint_device(sc.spp, sc.bounces, sc.p, d_w.data_ptr(), d_gs.data_ptr(), d_gm.data_ptr(), seed=seed,
                           stream=stream.cuda_stream)

    fwd()
    adj()
    t_f = min(timed(fwd) for _ in range(reps))
    t_a = min(timed(adj) for _ in range(reps))
    g_alb, g_th = sc.gradients(dimg, seed=seed)
    paths = H * W * sc.spp

    frng = np.random.default_rng(11)
    live_a = np.argwhere(g_alb != 0)
    live_t = np.argwhere(g_th != 0)
    out = []
    for k in range(n_fd):
        if frng.uniform() < 0.5 or len(live_t) == 0:
            i, j = (int(x) for x in live_a[frng.integers(len(live_a))])
            h, g = FD_H, g_alb[i, j]
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
            h, g = FD_H * th[i, j], g_th[i, j]
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
    gg = np.array([[o[3], o[4]] for o in out])
    floor = FD_FLOOR * float(np.sqrt(np.mean(gg[:, 1] ** 2)))
    rel = np.abs(gg[:, 0] - gg[:, 1]) / np.maximum(np.abs(gg[:, 1]), floor)
    rel_strict = np.abs(gg[:, 0] - gg[:, 1]) / np.maximum(np.abs(gg[:, 1]), 1e-300)
    worst = np.argsort(-rel)[:3]
    return {"forward_s": t_f, "adjoint_s": t_a, "cost_ratio": t_a / t_f,
            "forward_mpaths_s": paths / t_f / 1e6, "fd_params": n_fd,
            "fd": "central differences of the device renderer with the FP64 film, same seed (common random "
                  "numbers), h = %g (albedo samples) / %g x thickness; loss sum((I - T)^2) against a 1024-spp "
                  "target with hidden parameters" % (FD_H, FD_H),
            "rel_err": "|adjoint - fd| / max(|fd|, %g x RMS of the %d fds = %.3g)" % (FD_FLOOR, n_fd, floor),
            "within_2pct": int(np.sum(rel <= 0.02)), "within_2pct_without_floor": int(np.sum(rel_strict <= 0.02)),
            "rel_err_median": float(np.median(rel)), "rel_err_max": float(rel.max()),
            "worst": [list(out[w]) for w in worst],
            "drawn_from": "%d albedo samples, %d tiles with a non-zero adjoint gradient" % (len(live_a), len(live_t)),
            "workload": ADJ_DESC}


LARGE = dict(n_instances=256, width=3840, spp=256, bounces=32, p=0.8)
LARGE_DESC = ("large: 256 instances of a 65,536-triangle displaced UV sphere (16.8M instanced tris), 2-tri "
              "ground, 2 quad lights, 3840x2160, 256 spp, 32 bounces, p=0.8, 16 hero wavelengths 400-720 nm "
              "(80 bins); 16 tile jobs (4x4) of the frame in one batched launch; one adjoint pass (all "
              "albedo and thin-film IOR spectra, thicknesses, exponents)")


def run_large(spp=None, oracle_rows=2, oracle_spp=1024):
    """Config 5: the 4K frame as 16 tile jobs in one batched launch, the
    same frame as one plain render, one adjoint pass of it, and the RMSE of
    oracle_rows rows of the tiled frame against the reference's FP64 film
    at oracle_spp (the reference's own rows at the frame's spp beside it).
    Each is timed once, after a warm-up at 96 spp (tiles) and 32 spp
    (adjoint) that sizes the same buffers."""
    import numpy as np
    import torch

    from lambda_b200 import synth
    from lambda_b200.renderer import Context
    from lambda_b200.scene import flatten, load_nls
    w = dict(LARGE)
    if spp:
        w["spp"] = spp
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
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    ctx.render_batch_device([dict(t, spp=min(96, w["spp"])) for t in tiles], [d_tiles.data_ptr()] * 16,
                            stream=stream.cuda_stream)
    t_tiles = timed(lambda: ctx.render_batch_device(tiles, [d_tiles.data_ptr()] * 16, stream=stream.cuda_stream))
    t_plain = timed(lambda: ctx.render_device(w["spp"], w["bounces"], w["p"], d_out.data_ptr(), seed=3,
                                              stream=stream.cuda_stream))
    same = bool(torch.equal(d_out, d_tiles))
    wimg = torch.from_numpy(np.random.default_rng(5).standard_normal(H * W * 3).astype(np.float32)).cuda()
    n_spec = int(fs.scene.n_spectra) * int(fs.scene.spec.n_bins)
    d_gs = torch.zeros(n_spec, dtype=torch.float32, device="cuda")
    d_gm = torch.zeros(4 * int(fs.scene.n_materials), dtype=torch.float32, device="cuda")

    def adj(n_spp):
        ctx.adjoint_device(n_spp, w["bounces"], w["p"], wimg.data_ptr(), d_gs.data_ptr(), d_gm.data_ptr(), seed=3,
                           stream=stream.cuda_stream)
    adj(min(32, w["spp"]))
    t_adj = timed(lambda: adj(w["spp"]))
    out = {"value": paths / t_tiles / 1e6, "unit": UNIT, "seconds": t_tiles, "paths": paths,
           "plain_value": paths / t_plain / 1e6, "tiles_identical_to_plain": same,
           "adjoint_s": t_adj, "adjoint_cost_ratio": t_adj / t_plain,
           "gradient_nonzero": int((d_gs != 0).sum().item() + (d_gm != 0).sum().item()),
           "workload": LARGE_DESC}
    from oracle import refharness
    if oracle_rows and refharness.available(fast=True):
        img = d_tiles.cpu().numpy().reshape(H, W, 3).astype(np.float64)
        ref = refharness.RefScene(nls, fast=True)
        rows = [int(round(x)) for x in np.linspace(H * 0.3, H * 0.7, oracle_rows)]
        t0 = time.perf_counter()
        orc = np.stack([ref.render_rows(oracle_spp, w["bounces"], w["p"], r, r + 1, fp64=True,
                                        seed_base=W * H)[0] for r in rows])
        cref = np.stack([ref.render_rows(w["spp"], w["bounces"], w["p"], r, r + 1)[0] for r in rows])
        dev = image_stats(np.stack([img[H - 1 - r] for r in rows]), orc)
        cpu = image_stats(cref, orc)
        out["rmse"] = {"device": dev, "reference": cpu,
                       "ratio": [a / b for a, b in zip(dev["rel_rmse"], cpu["rel_rmse"])],
                       "rows": rows, "oracle_seconds": time.perf_counter() - t0,
                       "oracle": "reference FP64 film (oracle/_ref fast build), %d spp, seed base w*h, %d rows "
                                 "of the tiled 4K frame" % (oracle_spp, len(rows))}
    ctx.close()
    return out


BOX_DESC = ("box room: unit cube of 5 walls (10 tris; white 0.75, left 0.6 above 600 nm, right 0.6 on 500-560 nm), "
            "2 blocks (12 tris each), 0.25x0.25 ceiling quad light (blackbody 6500 K); 256x256, 16 spp, "
            "8 bounces, p=0.8, 4 hero wavelengths on 380-780 nm (81 bins)")
BOX = dict(width=256, spp=16, bounces=8, p=0.8)


def run_box_room(device, steps=20, warmup=3):
    """Config 1: the box room on the device (scene resident, CUDA events,
    L2 flushed between renders; and end to end through the C ABI), the
    reference built at the configuration's spectral setting
    (oracle/_ref/libref_k4_fast.so) on the host's cores for the whole
    frame, and the fixed-RMSE check against that build's FP64 film."""
    import numpy as np
    import torch

    from lambda_b200 import synth
    from lambda_b200.renderer import Context
    from lambda_b200.scene import SpectralConfig, flatten, load_nls
    root = os.path.join(tempfile.gettempdir(), "lgpu_bench", "box")
    nls = synth.box_room(root, width=BOX["width"])
    cfg = SpectralConfig(n_bins=81, lambda_inf=380.0, lambda_sup=780.0, hero_k=4)
    fs = flatten(load_nls(nls, cfg))
    ctx = Context(device)
    ctx.upload(fs)
    W, H = ctx.size
    spp, B, p = BOX["spp"], BOX["bounces"], BOX["p"]
    paths = W * H * spp
    d_out = torch.empty(W * H * 3, dtype=torch.float32, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    for k in range(warmup):
        ctx.render_device(spp, B, p, d_out.data_ptr(), seed=100 + k, stream=stream.cuda_stream)
    total = 0.0
    for k in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.render_device(spp, B, p, d_out.data_ptr(), seed=k, stream=stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1) / 1e3
    host = np.empty((H, W, 3), np.float32)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(steps):
        ctx.upload(fs)
        ctx.render(spp, B, p, seed=k, out=host)
    e2e_s = time.perf_counter() - t0
    launches = int(ctx.stats()["launches"])
    # the one-thread-per-pixel megakernel on the same frame (same paths)
    from lambda_b200 import _lib as L
    mega = 0.0
    for k in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.render_device(spp, B, p, d_out.data_ptr(), seed=k, flags=L.FLAG_MEGAKERNEL, stream=stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        mega += e0.elapsed_time(e1) / 1e3
    out = {"value": paths * steps / total / 1e6, "unit": UNIT, "ms_per_frame": total / steps * 1e3,
           "launches_per_frame": launches, "megakernel_value": paths * steps / mega / 1e6,
           "e2e": {"value": paths * steps / e2e_s / 1e6, "unit": UNIT,
                   "h2d_bytes_per_step": int(ctx.stats()["upload_bytes"]), "d2h_bytes_per_step": W * H * 12},
           "workload": BOX_DESC}
    from oracle import refharness
    if refharness.available(fast=True, k4=True):
        ref = refharness.RefScene(nls, fast=True, k4=True)
        ref.render_rows(spp, B, p, 0, H)
        reps = 3
        t0 = time.perf_counter()
        for _ in range(reps):
            ref.render_rows(spp, B, p, 0, H)
        v = paths * reps / (time.perf_counter() - t0) / 1e6
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": ref.L.ref_max_threads(), "kind": "reference",
                               "sample": "the whole frame (%d paths), reference built with 4 hero wavelengths, "
                                         "81 bins on 380-780 nm" % paths}
        out["vs_cpu"] = {"value": out["value"] / v, "e2e": out["e2e"]["value"] / v}
        out["rmse"] = rmse_check(ctx, dict(spp=spp, bounces=B, p=p), nls, d_out, stream, n_rows=H,
                                 oracle_spp=512, hi_spp=256, k4=True)
    ctx.close()
    return out


def image_stats(img, oracle):
    """Relative RMSE per channel against the oracle, and the bias: the mean
    per-pixel difference over its standard error (pixels draw independent
    streams) and the ratio of the means with its standard error."""
    import numpy as np
    d = (np.asarray(img, np.float64) - oracle).reshape(-1, 3)
    o = np.asarray(oracle, np.float64).reshape(-1, 3)
    se = d.std(axis=0, ddof=1) / np.sqrt(d.shape[0])
    om = o.mean(axis=0)
    rrmse = np.sqrt(np.mean(d ** 2, axis=0)) / np.sqrt(np.mean(o ** 2, axis=0))
    return {"rel_rmse": rrmse.tolist(), "t": (d.mean(axis=0) / se).tolist(),
            "mean_ratio": (1.0 + d.mean(axis=0) / om).tolist(), "mean_ratio_se": (se / om).tolist()}


def rmse_check(ctx, w, nls, d_out, stream, n_rows=24, oracle_spp=1024, hi_spp=512, k4=False):
    """Fixed-RMSE check against the reference itself: on n_rows scene rows
    spread over the frame, an FP64-film oracle rendered by the reference
    (oracle/_ref, fast build) at oracle_spp on streams disjoint from its
    own render (seed base w*h); the reference's own rows at the workload's
    spp (Renderer::render's streams); the device frame at that spp and at
    hi_spp.  Reports relative RMSE of both against the oracle, their ratio,
    and the device's and the reference's mean ratios to the oracle with
    standard errors."""
    import numpy as np
    import torch
    from oracle import refharness
    ref = refharness.RefScene(nls, fast=True, k4=k4)
    W, H = ctx.size
    spp, B, p = w["spp"], w["bounces"], w["p"]
    rows = sorted(set(int(round(x)) for x in np.linspace(0, H - 1, n_rows)))
    t0 = time.perf_counter()
    orc = np.stack([ref.render_rows(oracle_spp, B, p, r, r + 1, fp64=True, seed_base=W * H)[0] for r in rows])
    t_orc = time.perf_counter() - t0
    cref = np.stack([ref.render_rows(spp, B, p, r, r + 1)[0] for r in rows]).astype(np.float64)

    def device_rows(n_spp, seed):
        ctx.render_device(n_spp, B, p, d_out.data_ptr(), seed=seed, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        img = d_out.cpu().numpy().reshape(H, W, 3).astype(np.float64)
        return np.stack([img[H - 1 - r] for r in rows])  # scene row r is image row H - 1 - r

    dev = image_stats(device_rows(spp, 1), orc)
    cpu = image_stats(cref, orc)
    hi = image_stats(device_rows(hi_spp, 2), orc)
    return {"device": dev, "reference": cpu,
            "ratio": [a / b for a, b in zip(dev["rel_rmse"], cpu["rel_rmse"])],
            "device_%dspp" % hi_spp: {"t": hi["t"], "mean_ratio": hi["mean_ratio"],
                                       "mean_ratio_se": hi["mean_ratio_se"]},
            "rows": len(rows), "pixels": len(rows) * W, "oracle_seconds": t_orc,
            "oracle": "reference FP64 film (oracle/_ref fast build), %d spp, seed base w*h (streams disjoint "
                      "from Renderer::render's), %d rows spread over the frame" % (oracle_spp, len(rows)),
            "what": "relative RMSE per channel (R, G, B) at %d spp of the device frame and of the reference's "
                    "own render, both against the oracle; t = mean per-pixel difference / its standard error"
                    % spp}


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
    e2e_steps = max(1, min(args.steps, 10))
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
                   "readback) per step; the meshes' BVHs (the reference's and the traversal "
                   "tree) are built at scene load, as the reference builds its own (scene_build)"}
    scene_build = tree_build_times(sc)
    scene_build["e2e_with_traversal_tree_build"] = job_throughput(
        paths_per_step, 1, world, e2e_s * 1e3 / e2e_steps + scene_build["traversal_tree_ms"])

    c = counters[-1]
    launches_per_step = int(c["launches"])
    roofline = kernel_roofline(ctx, spp, B, p, stream, clk.get("sm_mhz"))

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generator)",
            "config": {"workload": workload_desc(w), "paths_per_step_per_gpu": paths_per_step,
                       "l2": "256 MB buffer written between timed steps",
                       "parallelism": "frame per GPU" if world > 1 else "single GPU"},
            "e2e": e2e, "scene_build": scene_build, "roofline": roofline, "clocks": clk,
            "gpu_launches": launches_per_step * args.steps,
            "mrays_per_s": world * c["rays"] * args.steps / (total_ms / 1e3) / 1e6}
    if rank == 0 and world == 1 and not args.no_baseline:
        # the reference's pixel loop on the host's cores, before the sections
        # below load those cores with oracle renders
        from oracle import refharness
        if refharness.available(fast=True):
            v, cores, sample = cpu_reference_sample(nls, w, args.ref_step_s)
            line["cpu_baseline"] = {"value": v / 1e6, "unit": UNIT, "cores": cores,
                                    "kind": "reference", "sample": sample}
            line["rmse"] = rmse_check(ctx, w, nls, d_out, stream)
    if rank == 0 and world == 1 and not args.no_batch:
        line["batched"] = run_batched(Context, local)
    if rank == 0 and world == 1 and not args.no_adjoint:
        line["adjoint"] = run_adjoint(local)
    if rank == 0 and world == 1 and not args.no_box:
        line["box_room"] = run_box_room(local)
    if rank == 0 and world == 1 and not args.no_large:
        line["large"] = run_large()
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


def tree_build_times(sc, reps=3):
    """Host time of the two BVH builds of the scene's largest mesh (median
    of reps): the reference's tree (lgpu_build_bvh, bvh::build) and the
    traversal tree (lgpu_build_traversal_bvh), both run by the loader."""
    m = max(sc.meshes, key=lambda x: x.F.shape[0])
    out = {"faces": int(m.F.shape[0]), "threads": os.cpu_count()}
    for key, fn in (("reference_tree_ms", "lgpu_build_bvh"), ("traversal_tree_ms", "lgpu_build_traversal_bvh")):
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            m._tree(fn)
            ts.append((time.perf_counter() - t0) * 1e3)
        out[key] = float(statistics.median(ts))
    return out


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
                    help="only the large configuration (4K, 16 tile jobs, one adjoint pass)")
    ap.add_argument("--no-large", action="store_true", help="skip the large configuration")
    ap.add_argument("--no-box", action="store_true", help="skip the box-room configuration")
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
        big = run_large(args.spp)
        line = {"metric": METRIC, "value": big["value"], "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": 1,
                "ms_per_step": big["seconds"] * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
                "config": {"workload": LARGE_DESC, "paths": big["paths"]}, "large": big}
        print(json.dumps(line))
        return 0
    return run_device(args, w)


if __name__ == "__main__":
    sys.exit(main())
