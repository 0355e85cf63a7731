"""Benchmark: paths/s of the FP32 wavefront path integrator on the 1080p
mesh + env-map workload (1920x1080, 256 spp, max depth 16, rr depth 3;
1,310,720-triangle displaced icosphere + 200 random spheres, 1024x512 sky +
sun env map; seeded synthetic scene).

One step = one full render of that frame.  On N GPUs (one process each,
torchrun) the frame is split by film rows: rank r renders rows r, r + N,
r + 2N, ... with every pixel's RNG stream unchanged, and one NCCL all-gather
of the padded f64 film rows assembles the whole film (strong scaling: the
total work per step is one frame whatever N is).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the CPU f64 restatement of the reference renderer
(the reference is Rust and cannot be built here) on the host cores, on a
bounded sample of rows of the same frame.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "paths/s at 1080p, FP32 wavefront (mesh+env workload)"
UNIT = "paths/s"
WORKLOAD = ("mesh_env_1080p: 1920x1080, 256 spp, max_depth 16, rr_depth 3, 1,310,720-triangle displaced icosphere "
            "+ 200 spheres, 1024x512 float32 sky+sun env map")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--spp", type=int, default=256)
    p.add_argument("--width", type=int, default=1920)
    p.add_argument("--height", type=int, default=1080)
    p.add_argument("--subdiv", type=int, default=8)
    p.add_argument("--plain-spp", type=int, default=8, help="spp of the plain f64 comparison render")
    p.add_argument("--profile-spp", type=int, default=0,
                   help="spp of the instrumented roofline pass (0 = same as --spp, so the schedule matches)")
    p.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of a baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--rmse-spp", type=int, default=256, help="spp of the equal-RMSE comparison renders")
    p.add_argument("--no-rmse", action="store_true", help="skip the comparison against the ground truth")
    p.add_argument("--adjoint-steps", type=int, default=5, help="timed inverse-rendering steps (0 = skip)")
    p.add_argument("--adjoint-size", type=int, default=512, help="film edge of the inverse-rendering workload")
    p.add_argument("--adjoint-spp", type=int, default=64, help="forward and adjoint spp of the inverse-rendering step")
    p.add_argument("--adjoint-only", action="store_true", help="run only the inverse-rendering leg (profiling)")
    p.add_argument("--batch-scenes", type=int, default=64, help="scenes of the batch workload (0 = skip)")
    p.add_argument("--batch-only", action="store_true", help="run only the batch leg")
    p.add_argument("--adaptive-spp", type=int, default=4096, help="max spp of the adaptive Cornell frame (0 = skip)")
    p.add_argument("--adaptive-only", action="store_true", help="run only the adaptive Cornell leg")
    p.add_argument("--quick", action="store_true", help="small frame for a functional check")
    p.add_argument("--bvh-reps", type=int, default=5, help="timed device BVH builds of the workload mesh (0 = skip)")
    p.add_argument("--bvh-only", action="store_true", help="run only the BVH build leg")
    p.add_argument("--frame-only", action="store_true",
                   help="render the workload frame --warmup + --steps times and print per-frame times (profiling, "
                        "A/B of TPT_* settings); no other legs")
    p.add_argument("--no-cpu-configs", action="store_true", help="skip the CPU baselines of the other configs")
    return p.parse_args()


# ---- clocks ------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---- helpers ----------------------------------------------------------------------------------------------
def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def frame_only(args):
    """Renders the workload frame --warmup + --steps times through
    tpt_render_device and prints each timed frame's device ms (profiling and
    A/B runs of the TPT_* settings)."""
    import torch

    from tinypt_b200 import _abi
    from tinypt_b200.render import DeviceScene

    torch.cuda.set_device(0)
    n = args.width * args.height
    cfg = cfg_for(args, _abi.TPT_MODE_WAVEFRONT_FP32, args.spp, 1)
    with DeviceScene(build_workload(args)) as ds:
        acc = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
        acc_w = torch.zeros(n, dtype=torch.float64, device="cuda")
        ms, st = [], None
        for i in range(args.warmup + args.steps):
            st = ds.render_device(cfg, acc.data_ptr(), acc_w.data_ptr())
            if i >= args.warmup:
                ms.append(st.render_ms)
    best = min(ms) if ms else float("nan")
    print(json.dumps({"frame_only": {
        "width": args.width, "height": args.height, "spp": args.spp, "ms": [round(x, 3) for x in ms],
        "paths_per_s_best": n * args.spp / (best / 1000.0), "paths_per_s_median": n * args.spp / (statistics.median(ms) / 1000.0),
        "iterations": st.iterations if st else 0, "rays": st.rays if st else 0,
        "rays_closest_traced": (st.rays_closest - st.sky_samples) if st else 0,
        "rays_shadow": st.rays_shadow if st else 0, "culled_samples": st.sky_samples if st else 0,
        "task_spp": st.task_spp if st else 0, "pool_slots": st.pool_slots if st else 0,
        "kernel_launches": st.kernel_launches if st else 0,
        "env": {k: v for k, v in os.environ.items() if k.startswith("TPT_")}}}), flush=True)


def probe_bandwidth(nbytes: int, reps: int):
    """Read bandwidth (GB/s) of a buffer of nbytes streamed reps times with
    L1 bypassed (tpt_probe_read_bandwidth, current device); None on error."""
    import ctypes as C

    from tinypt_b200 import _abi

    g = C.c_double()
    rc = _abi.lib().tpt_probe_read_bandwidth(nbytes, reps, C.byref(g))
    return g.value if rc == 0 else None


def ncu_traffic_per_ray():
    """DRAM bytes per traced closest-hit ray of k_trace<closest> from the
    committed ncu summary (a saturated launch of a reduced case), if any."""
    p = ROOT / "profiles" / "k_trace_closest_mesh_env_1080p.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get("dram_bytes_per_traced_ray")
        except Exception:
            return None
    return None


def build_workload(args, rank=0):
    from tinypt_b200 import scenes

    if args.quick:
        scene = scenes.mesh_env_scene(args.width, args.height, subdiv=5, n_spheres=200, env_w=256, env_h=128)
    else:
        scene = scenes.mesh_env_scene(args.width, args.height, subdiv=args.subdiv)
    return scene


def cfg_for(args, mode, spp, seed):
    from tinypt_b200.scene import RenderConfig

    return RenderConfig(width=args.width, height=args.height, spp=spp, max_bounces=16, rr_start=3, seed=seed, mode=mode)


# ---- CPU baseline: the oracle on the host cores --------------------------------------------------------------
def cpu_sample(args, scene, target_seconds, threads):
    """Times the f64 CPU restatement on whole frames of the workload: one
    1-spp frame to calibrate, then one frame at the spp that fills about
    target_seconds; returns (paths/s, description, seconds)."""
    from oracle import oracle
    from tinypt_b200 import _abi

    with oracle.OracleScene(scene) as os_:
        t0 = time.perf_counter()
        os_.render(cfg_for(args, _abi.TPT_MODE_PLAIN_F64, 1, 7), threads=threads)
        t_frame = max(time.perf_counter() - t0, 1e-3)
        spp = max(1, int(round(target_seconds / t_frame)))
        t0 = time.perf_counter()
        os_.render(cfg_for(args, _abi.TPT_MODE_PLAIN_F64, spp, 1), threads=threads)
        dt = time.perf_counter() - t0
    paths = args.width * args.height * spp
    desc = (f"the whole {args.width}x{args.height} frame at {spp} spp ({paths} paths, {dt:.1f} s), "
            f"C++ f64 restatement of the reference renderer")
    return paths / dt, desc, dt


def cpu_config_baselines(threads: int):
    """The oracle (C++ f64 restatement of the reference renderer) on the other
    configs, on the host cores, each a bounded sample timed like the
    reference's own `Done in` line (render only; scene and BVH builds
    excluded, render.rs:263).  Returns {config: {paths_per_s, ...}}."""
    import concurrent.futures as cf
    import dataclasses

    from oracle import oracle
    from tinypt_b200 import _abi, scenes
    from tinypt_b200.scene import RenderConfig

    PL = _abi.TPT_MODE_PLAIN_F64
    out = {}

    def timed(scene, cfg, label, note):
        with oracle.OracleScene(scene) as os_:
            t0 = time.perf_counter()
            _, w, _, _ = os_.render(cfg, threads=threads)
            dt = time.perf_counter() - t0
        paths = float(w.sum())
        out[label] = {"paths_per_s": paths / dt, "paths": paths, "seconds": dt, "cores": threads, "kind": "port",
                      "sample": note}

    # C1: the whole config (256x256, 64 spp, depth 8)
    timed(scenes.sphere_scene(256, 256), scenes.sphere_scene_config(256, 256, 64), "C1",
          "sphere scene, the whole config: 256x256, 64 spp, max_depth 8, rr 3, seed 1")
    # C4: the Cornell frame at 960x540, adaptive with at most 16 spp (a reduced
    # sample of the 1080p, 4096-spp config; paths/s, not the image, is compared)
    c4 = dataclasses.replace(scenes.cornell_config(960, 540, spp=16), seed=1)
    timed(scenes.cornell_scene(960, 540), c4, "C4",
          "Cornell + 262,144-triangle GGX mesh + absorbing dielectric, 960x540, adaptive (thr 0.01, min 8, max 16 "
          "spp), max_depth 32")
    # C5: the forward half of the inverse-rendering step (512x512, depth 8), at
    # 16 of its 64 spp (paths/s does not depend on spp for a uniform render)
    c5 = RenderConfig(width=512, height=512, spp=16, max_bounces=8, rr_start=3, seed=1, mode=PL)
    timed(scenes.inverse_scene(512, 512), c5, "C5",
          "inverse-rendering scene, forward only (the reference has no adjoint): 512x512, 16 of the config's 64 "
          "spp, max_depth 8")
    # C3: the 64 batch scenes one after another, each at 1 spp of its own film
    work = scenes.batch_workload(64)
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:  # scene + BVH builds in parallel (untimed)
        built = list(ex.map(lambda sc: oracle.OracleScene(sc[0]), work))
    t0 = time.perf_counter()
    paths = 0.0
    for os_, (_, c) in zip(built, work):
        _, w, _, _ = os_.render(dataclasses.replace(c, spp=1, mode=PL), threads=threads)
        paths += float(w.sum())
    dt = time.perf_counter() - t0
    for os_ in built:
        os_.close()
    out["C3"] = {"paths_per_s": paths / dt, "paths": paths, "seconds": dt, "cores": threads, "kind": "port",
                 "sample": "the 64 batch scenes rendered one after another, each at 1 spp of its own film "
                           "(128-1008 px square), max_depth 12"}
    return out


# ---- reference arm -------------------------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    scene = build_workload(args)
    from oracle import oracle
    from tinypt_b200 import _abi

    with oracle.OracleScene(scene) as os_:
        t0 = time.perf_counter()
        os_.render(cfg_for(args, _abi.TPT_MODE_PLAIN_F64, 1, 7), threads=threads)
        t_frame = max(time.perf_counter() - t0, 1e-3)
        per_step = max(4.0, min(20.0, 150.0 / max(args.steps + args.warmup, 1)))
        spp = max(1, int(round(per_step / t_frame)))
        cfg = cfg_for(args, _abi.TPT_MODE_PLAIN_F64, spp, 1)

        def step():
            os_.render(cfg, threads=threads)

        for _ in range(args.warmup):
            step()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
        dt = time.perf_counter() - t0
    paths = args.width * args.height * spp * args.steps
    value = paths / dt
    sample = (f"the whole {args.width}x{args.height} mesh_env frame at {spp} spp per step; C++ f64 restatement "
              f"of the reference renderer (the Rust reference is not buildable: no toolchain)")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * dt / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "parallelism": f"{threads} host threads"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- precision against the ground truth ----------------------------------------------------------------------
def equal_rmse(args, ds, wf_value, plain_value):
    """Renders the 240x135 film of the same scene (same camera and aspect, so
    the 1080p scene handle serves) with both forms, measures each image's
    error against the committed 65536-spp plain-f64 ground truth, and turns
    the MSE ratio at equal spp and the 1080p throughputs into the equal-RMSE
    speed-up of the FP32 wavefront form over the plain f64 form."""
    import torch

    from tinypt_b200 import _abi, precision
    from tinypt_b200.scene import RenderConfig

    if not precision.TRUTH_FILE.exists():
        return {"unavailable": "ground-truth fixture missing"}
    truth, meta = precision.load_truth()
    w, h = precision.TRUTH_WIDTH, precision.TRUTH_HEIGHT
    n = w * h
    acc = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    acc_w = torch.zeros(n, dtype=torch.float64, device="cuda")

    def errors(mode, spp, seeds):
        rows = []
        for seed in seeds:
            cfg = RenderConfig(width=w, height=h, spp=spp, max_bounces=16, rr_start=3, seed=seed, mode=mode)
            st = ds.render_device(cfg, acc.data_ptr(), acc_w.data_ptr())
            img = (acc.view(n, 3) / acc_w.clamp(min=1.0)[:, None]).cpu().numpy()
            e = precision.image_error(img, truth)
            e["flags"] = st.device_flags
            rows.append(e)
        return {"spp": spp, "renders": len(rows), "mse": statistics.fmean(r["mse"] for r in rows),
                "rmse": statistics.fmean(r["rmse"] for r in rows),
                "rel_rmse": statistics.fmean(r["rel_rmse"] for r in rows),
                "mean_rel_err": statistics.fmean(r["mean_rel_err"] for r in rows),
                "device_flags": max(r["flags"] for r in rows)}

    wf, pl = _abi.TPT_MODE_WAVEFRONT_FP32, _abi.TPT_MODE_PLAIN_F64
    s = args.rmse_spp
    res = {"film": f"{w}x{h} of the same scene and camera",
           "truth": f"plain f64 GPU form, {meta['spp']} spp (seeds {meta['seeds'][0]}..{meta['seeds'][-1]})",
           "wavefront_fp32": errors(wf, s, list(range(11, 19))), "plain_f64": errors(pl, s, list(range(21, 29))),
           "wavefront_fp32_16x": errors(wf, 16 * s, [15]), "plain_f64_16x": errors(pl, 16 * s, [25])}
    res["mse_ratio_plain_over_wavefront"] = res["plain_f64"]["mse"] / res["wavefront_fp32"]["mse"]
    res["speedup"] = precision.equal_rmse_speedup(wf_value, res["wavefront_fp32"]["mse"], plain_value,
                                                  res["plain_f64"]["mse"])
    res["definition"] = ("speedup = (paths/s wavefront / paths/s plain, both at 1080p, 1 GPU) x "
                         "(MSE plain / MSE wavefront at equal spp vs the ground truth)")
    return res


# ---- adjoint: inverse-rendering step -------------------------------------------------------------------------
def adjoint_leg(args):
    """One optimisation step of the inverse-rendering workload: forward
    render (64 spp) -> L2 loss gradient against the target -> adjoint render
    (64 spp, path replay) -> parameter update.  512x512 film, 262,144-triangle
    heightfield in 16 GGX material groups (64 parameters), 512x256 env map,
    max_depth 8.  The target is rendered from the seeded ground-truth
    parameters; optimisation starts from perturbed ones."""
    import torch

    from tinypt_b200 import _abi, autodiff, scenes
    from tinypt_b200.render import DeviceScene
    from tinypt_b200.scene import RenderConfig

    w = h = args.adjoint_size
    spp = args.adjoint_spp
    truth = scenes.inverse_params()
    start = np.clip(truth + np.random.default_rng(4).normal(0.0, 0.12, truth.shape), 0.05, 0.95)
    scene = scenes.inverse_scene(w, h)
    base = scene.mats

    def cfg(spp, seed):
        return RenderConfig(width=w, height=h, spp=spp, max_bounces=8, rr_start=3, seed=seed,
                            mode=_abi.TPT_MODE_WAVEFRONT_FP32)

    with DeviceScene(scene) as ds:
        target = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
        ds.render_forward(cfg(256, 1), target.data_ptr())
        img = torch.empty_like(target)
        grad = torch.empty(4 * len(base), dtype=torch.float64, device="cuda")
        params = start.copy()
        m = np.zeros_like(params)
        v = np.zeros_like(params)
        losses, fwd_ms, bwd_ms = [], [], []

        def step(it):
            ds.set_materials(autodiff.materials_with(base, params))
            fs = ds.render_forward(cfg(spp, 1000 + it), img.data_ptr())
            diff = img - target
            loss = float((diff * diff).mean())
            dimg = (2.0 / diff.numel()) * diff
            bs = ds.render_backward(cfg(spp, 2000 + it), dimg.data_ptr(), grad.data_ptr())
            g = grad.view(-1, 4).cpu().numpy()
            # Adam on the 64 parameters (host; 64 numbers)
            m[:] = 0.9 * m + 0.1 * g
            v[:] = 0.999 * v + 0.001 * g * g
            params[:] = np.clip(params - 0.02 * (m / (1 - 0.9 ** (it + 1))) /
                                (np.sqrt(v / (1 - 0.999 ** (it + 1))) + 1e-8), 0.02, 0.98)
            return loss, fs.render_ms, bs.render_ms

        for it in range(2):
            step(it)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for it in range(2, 2 + args.adjoint_steps):
            loss, f, b = step(it)
            losses.append(loss)
            fwd_ms.append(f)
            bwd_ms.append(b)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    k = args.adjoint_steps
    paths = w * h * spp
    return {
        "workload": f"inverse rendering: {w}x{h}, 262,144-triangle heightfield in 16 GGX material groups "
                    f"(64 parameters), 512x256 env, {spp} spp forward + {spp} spp adjoint, max_depth 8",
        "ms_per_step": 1000.0 * dt / k, "steps": k,
        "forward_ms": statistics.fmean(fwd_ms), "backward_ms": statistics.fmean(bwd_ms),
        "backward_paths_per_s": paths / (statistics.fmean(bwd_ms) / 1000.0),
        "loss": [round(x, 6) for x in losses],
        "param_error": {"start": float(np.abs(start - truth).mean()), "end": float(np.abs(params - truth).mean())},
        "timing": "host wall clock around synchronous API calls (device idle between); forward/backward ms from "
                  "CUDA events inside the library",
    }


# ---- batch: many scenes in one call ---------------------------------------------------------------------------
# the library's threshold for a batch job to render alone (tpt_batch_render_device)
BATCH_ALONE_PATHS = 16 << 20


def batch_leg(args):
    """The batch workload: 64 seeded scenes (displaced icospheres and boxes,
    log-uniform 1k-500k triangles, one area light each), square films
    log-uniform 128-1024 px and spp log-uniform 16-256, max_depth 12.  The
    schedule is picked by the library's autotuner; the batch then renders in
    one call: jobs of at least 16 Mi paths alone with the single-render
    schedule, the others in one wavefront loop.  Two unbatched times: the
    same jobs one after another through the same handle, and each scene
    through the single-render entry."""
    import torch

    from tinypt_b200 import scenes
    from tinypt_b200.render import BatchScenes

    work = scenes.batch_workload(args.batch_scenes)
    t0 = time.perf_counter()
    bs = BatchScenes([s for s, _ in work])
    build_s = time.perf_counter() - t0
    films = [(torch.empty(3 * c.film_pixels, dtype=torch.float64, device="cuda"),
              torch.empty(c.film_pixels, dtype=torch.float64, device="cuda")) for _, c in work]
    jobs = [(k, c, a.data_ptr(), w.data_ptr()) for k, ((_, c), (a, w)) in enumerate(zip(work, films))]
    paths = sum(c.film_pixels * c.spp for _, c in work)
    t0 = time.perf_counter()
    tuning, trials = bs.autotune(jobs)
    tune_s = time.perf_counter() - t0
    bs.render(jobs, tuning=tuning)  # warm-up
    batch_ms = [bs.render(jobs, tuning=tuning).render_ms for _ in range(2)]
    # one job per launch, each job under the batch's tuning or the default
    # schedule, whichever is faster for it (tasks long enough to fill the
    # pool for 64 jobs leave one job's pool half empty)
    seq_tuned = [bs.render([j], tuning=tuning).render_ms for j in jobs]
    seq_default = [bs.render([j]).render_ms for j in jobs]
    default_ms = bs.render(jobs).render_ms
    bs.close()
    # and each scene through the single-render entry (tpt_render_device,
    # its own handle; camera culling applies there), the second render timed
    from tinypt_b200.render import DeviceScene

    single = []
    for (scene, c), (a, w) in zip(work, films):
        with DeviceScene(scene) as ds:
            ds.render_device(c, a.data_ptr(), w.data_ptr())
            single.append(ds.render_device(c, a.data_ptr(), w.data_ptr()).render_ms)
    seq_ms = sum(min(a, b) for a, b in zip(seq_tuned, seq_default))
    tris = [sum(m.n_tris for m in s.world.meshes) for s, _ in work]
    res = [c.width for _, c in work]
    spp = [c.spp for _, c in work]
    best = min(batch_ms)
    alone_paths = int(os.environ.get("TPT_BATCH_ALONE_PATHS", BATCH_ALONE_PATHS))
    n_alone = sum(1 for _, c in work if alone_paths > 0 and c.film_pixels * c.spp >= alone_paths)
    return {
        "workload": f"{len(work)} scenes, {min(tris)}-{max(tris)} triangles, films {min(res)}-{max(res)} px square, "
                    f"{min(spp)}-{max(spp)} spp, max_depth 12, one call: {n_alone} jobs of >= {alone_paths} paths "
                    f"alone with the single-render schedule, {len(work) - n_alone} in one wavefront loop",
        "paths": paths, "ms": best, "paths_per_s": paths / (best / 1000.0),
        "one_job_at_a_time_ms": seq_ms, "speedup_vs_one_at_a_time": seq_ms / best,
        "one_job_at_a_time_scope": ("each job alone through the batch handle, under the batch's tuning or the "
                                    "default schedule, per job the faster"),
        "one_job_at_a_time_tuned_ms": sum(seq_tuned), "one_job_at_a_time_default_ms": sum(seq_default),
        "single_renders_ms": sum(single), "speedup_vs_single_renders": sum(single) / best,
        "single_renders_scope": "each scene through tpt_render_device (own handle, its own schedule and culling)",
        "default_schedule_ms": default_ms,
        "tuning": {"pool_slots": tuning[0], "task_spp": tuning[1], "trace_chunk": tuning[2],
                   "shade_ctas": tuning[3]},
        "autotune_trials": len(trials), "autotune_s": tune_s, "build_s": build_s,
        "triangles_total": int(sum(tris)),
    }


def small_batch_leg():
    """Where batching pays: 64 small seeded scenes (1k-50k triangles, films
    32-96 px square, 4-16 spp, max_depth 12) in one autotuned launch,
    against the same scenes through tpt_render_device one after another
    (each scene's second render timed)."""
    import torch

    from tinypt_b200 import scenes
    from tinypt_b200.render import BatchScenes, DeviceScene

    work = scenes.batch_workload(64, seed=5, tri_range=(1_000, 50_000), res_range=(32, 96), spp_range=(4, 16))
    films = [(torch.empty(3 * c.film_pixels, dtype=torch.float64, device="cuda"),
              torch.empty(c.film_pixels, dtype=torch.float64, device="cuda")) for _, c in work]
    jobs = [(k, c, a.data_ptr(), w.data_ptr()) for k, ((_, c), (a, w)) in enumerate(zip(work, films))]
    paths = sum(c.film_pixels * c.spp for _, c in work)
    with BatchScenes([s for s, _ in work]) as bs:
        tuning, _ = bs.autotune(jobs)
        bs.render(jobs, tuning=tuning)
        best = min(bs.render(jobs, tuning=tuning).render_ms for _ in range(3))
    single = 0.0
    for (scene, c), (a, w) in zip(work, films):
        with DeviceScene(scene) as ds:
            ds.render_device(c, a.data_ptr(), w.data_ptr())
            single += ds.render_device(c, a.data_ptr(), w.data_ptr()).render_ms
    return {"workload": "64 scenes, 1k-50k triangles, films 32-96 px square, 4-16 spp, max_depth 12",
            "paths": paths, "ms": best, "paths_per_s": paths / (best / 1000.0), "single_renders_ms": single,
            "speedup_vs_single_renders": single / best}


# ---- adaptive sampling: Cornell box, max 4096 spp -------------------------------------------------------------
def adaptive_leg(args):
    """The adaptive-sampling workload: Cornell box + 262,144-triangle GGX
    mesh + absorbing dielectric sphere, 1920x1080, adaptive stop at relative
    sample standard deviation 0.01 (after 8 samples), at most 4096 spp,
    max_depth 32.  The 1080p frame is timed once; the error against the
    65536-spp f64 ground truth is measured on the 160x90 film of the same
    scene, for the adaptive render and for a uniform render with the same
    mean spp."""
    import dataclasses

    import torch

    from tinypt_b200 import precision, scenes
    from tinypt_b200.render import DeviceScene

    out = {}
    cfg = scenes.cornell_config(spp=args.adaptive_spp)
    with DeviceScene(scenes.cornell_scene(1920, 1080)) as ds:
        n = 1920 * 1080
        acc = torch.empty(3 * n, dtype=torch.float64, device="cuda")
        w = torch.empty(n, dtype=torch.float64, device="cuda")
        st = ds.render_device(cfg, acc.data_ptr(), w.data_ptr())
        ww = w.cpu().numpy()
    out.update({"workload": "Cornell box + 262,144-triangle GGX mesh + absorbing dielectric, 1920x1080, adaptive "
                            f"(rel. sample std < 0.01 after 8, max {cfg.spp} spp), max_depth 32",
                "ms": st.render_ms, "paths": st.paths, "paths_per_s": st.paths / (st.render_ms / 1000.0),
                "mean_spp": float(ww.mean()), "pixels_stopped_early": float((ww < cfg.spp).mean()),
                "iterations": st.iterations})
    if precision.CORNELL_TRUTH_FILE.exists():
        truth, meta = precision.load_truth(precision.CORNELL_TRUTH_FILE)
        cw, ch = precision.CORNELL_WIDTH, precision.CORNELL_HEIGHT
        small = dataclasses.replace(cfg, width=cw, height=ch, seed=7)
        with DeviceScene(scenes.cornell_scene(cw, ch)) as ds:
            n = cw * ch
            acc = torch.empty(3 * n, dtype=torch.float64, device="cuda")
            w = torch.empty(n, dtype=torch.float64, device="cuda")
            ds.render_device(small, acc.data_ptr(), w.data_ptr())
            img = (acc.view(n, 3) / w.clamp(min=1.0)[:, None]).cpu().numpy()
            spp_px = w.cpu().numpy()
            mean_spp = float(spp_px.mean())
            e_ad = precision.image_error(img, truth)
            # the reference's rule stops a pixel whose first 8 samples are equal: all-zero
            # samples in a dim region end the pixel at 0 although its true value is not 0
            e_ad["pixels_stopped_on_zero_samples"] = int(((spp_px <= small.adaptive_min_spp)
                                                          & (img.max(axis=1) == 0.0)
                                                          & (truth.max(axis=1) > 0.0)).sum())
            uni = dataclasses.replace(small, adaptive_enabled=False, spp=max(1, int(round(mean_spp))))
            ds.render_device(uni, acc.data_ptr(), w.data_ptr())
            img_u = (acc.view(n, 3) / w.clamp(min=1.0)[:, None]).cpu().numpy()
            e_un = precision.image_error(img_u, truth)
        out["error_vs_truth"] = {
            "film": f"{cw}x{ch} of the same scene and camera",
            "truth": f"plain f64 GPU form, {meta['spp']} spp",
            "adaptive": {**e_ad, "mean_spp": mean_spp}, "uniform_same_mean_spp": {**e_un, "spp": uni.spp}}
    return out


# ---- our arm ------------------------------------------------------------------------------------------------
def bvh_leg(args, scene):
    """Build time of the workload's mesh BVH: the device builder (median of
    --bvh-reps calls through the C ABI, host mesh in and host tree out) and the
    host builder (one call); both trees must be identical."""
    import numpy as np

    from tinypt_b200 import bvh

    mesh = scene.world.meshes[0]
    bvh.build(mesh, device=True)  # warm-up: context, allocator
    times = []
    for _ in range(args.bvh_reps):
        t0 = time.perf_counter()
        dev = bvh.build(mesh, device=True)
        times.append(time.perf_counter() - t0)
    t0 = time.perf_counter()
    host = bvh.build(mesh, device=False)
    host_s = time.perf_counter() - t0
    same = (dev.bbox.tobytes() == host.bbox.tobytes() and np.array_equal(dev.left_right, host.left_right)
            and np.array_equal(dev.start_count, host.start_count) and np.array_equal(dev.indices, host.indices))
    dev_s = float(np.median(times))
    return {"mesh": f"displaced icosphere, {mesh.n_tris} triangles", "nodes": dev.n_nodes,
            "device_ms": 1e3 * dev_s, "host_ms": 1e3 * host_s, "speedup": host_s / dev_s, "identical": bool(same),
            "timing": "wall clock around tpt_bvh_build_device / tpt_bvh_build_host, host arrays in and out"}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from tinypt_b200 import _abi, multigpu
    from tinypt_b200.render import DeviceScene

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    scene = build_workload(args, rank)
    n_px = args.width * args.height
    ds = DeviceScene(scene)
    acc = torch.zeros(3 * n_px, dtype=torch.float64, device=dev)
    acc_w = torch.zeros(n_px, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    cfg = cfg_for(args, _abi.TPT_MODE_WAVEFRONT_FP32, args.spp, 1)
    # N > 1: this rank's interleaved rows of the frame, then one all-gather of
    # the padded f64 rows (acc rgb + acc_w) into the whole film on every rank
    shard = multigpu.shard_config(cfg, rank, world)
    rows = shard.film_rows
    s_acc = torch.zeros(3 * rows * args.width, dtype=torch.float64, device=dev)
    s_w = torch.zeros(rows * args.width, dtype=torch.float64, device=dev)
    exchange = multigpu.ShardGather(args.width, args.height, rank, world, device=dev)

    def step():
        if world == 1:
            return ds.render_device(cfg, acc.data_ptr(), acc_w.data_ptr())
        st = ds.render_device(shard, s_acc.data_ptr(), s_w.data_ptr())
        exchange.gather(s_acc, s_w, acc, acc_w)
        return st

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- timed region: exactly K steps between barrier + synchronize
    launches = 0
    stats = []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        barrier()
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(args.steps):
            flush.fill_(1)  # L2 flush between steps (256 MiB write)
            st = step()
            stats.append(st)
            # the library's own count: camera culling (7) and the sky kernel,
            # the pool start, 8 kernels per iteration of the device-side loop,
            # the drain's tail kernel, the merge of the task sums
            launches += st.kernel_launches
        ev1.record()
        torch.cuda.synchronize()
        barrier()
    ms_local = ev0.elapsed_time(ev1)
    t = torch.tensor([ms_local], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    paths_per_step = n_px * args.spp  # one frame per step, whatever the number of GPUs
    value = paths_per_step * args.steps / (ms / 1000.0)
    rays = torch.tensor([float(sum(s.rays for s in stats)), float(sum(s.sky_samples for s in stats))],
                        dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(rays)
    rays_total, rays_culled = (float(x) for x in rays.tolist())

    # ---- end to end through the public API with host buffers: tpt_render on
    # one GPU; on N GPUs multigpu.render_sharded (rows + all-gather) and the
    # whole film read back to pinned host memory on rank 0
    host_acc = torch.empty(3 * n_px, dtype=torch.float64).pin_memory()
    host_w = torch.empty(n_px, dtype=torch.float64).pin_memory()
    e2e_steps = max(1, min(args.steps, 2))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        if world == 1:
            ds.render(cfg, host_acc.numpy(), host_w.numpy())
        else:
            f_acc, f_w = multigpu.render_sharded(ds, cfg)
            if rank == 0:
                host_acc.copy_(f_acc.reshape(-1))
                host_w.copy_(f_w.reshape(-1))
            torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    tt = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    e2e_value = n_px * args.spp * e2e_steps / float(tt.item())

    if rank != 0:
        ds.close()
        return

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD if not args.quick else "quick functional check (reduced scene)",
                   "width": args.width, "height": args.height, "spp": args.spp,
                   "parallelism": (f"strong: one frame per step split by film rows over {world} GPU(s) "
                                   "(rank r renders rows r, r+N, ...), NCCL all-gather of the f64 film rows")
                   if world > 1 else "1 GPU, one frame per step",
                   "l2": "flushed between steps (256 MiB write)", "accumulation": "f64"},
        # camera rays of culled pixels count as rays (their closest hit, none,
        # is decided by the frustum test); rays_traced_per_s leaves them out
        "rays_per_s": rays_total * 1.0 / (ms / 1000.0),
        "rays_traced_per_s": (rays_total - rays_culled) / (ms / 1000.0),
        "gpu_launches": launches,
        "camera_culled_share": stats[-1].sky_samples / max(stats[-1].paths, 1),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 64,
                "d2h_bytes_per_step": 4 * 8 * n_px,
                "api": "tpt_render (host output buffers; film copied device->host each step)" if world == 1 else
                       "multigpu.render_sharded (rows + NCCL all-gather), whole film read back on rank 0"},
    }

    # ---- plain f64 GPU form on the same frame (comparison, not the headline)
    plain_cfg = cfg_for(args, _abi.TPT_MODE_PLAIN_F64, args.plain_spp, 1)
    ds.render_device(plain_cfg, acc.data_ptr(), acc_w.data_ptr())
    torch.cuda.synchronize()
    pst = ds.render_device(plain_cfg, acc.data_ptr(), acc_w.data_ptr())
    plain_value = n_px * args.plain_spp / (pst.render_ms / 1000.0)
    out["plain_f64"] = {"value": plain_value, "unit": UNIT, "spp": args.plain_spp, "ms": pst.render_ms}
    out["speedup_vs_plain_f64_same_spp"] = value / world / plain_value  # per GPU

    # ---- precision: both forms against the 65536-spp f64 ground truth
    if not args.quick and args.subdiv == 8 and not args.no_rmse:
        out["equal_rmse"] = equal_rmse(args, ds, value / world, plain_value)

    # ---- roofline of the dominant kernel (k_trace<closest>, closest-hit traversal)
    prof_cfg = cfg_for(args, _abi.TPT_MODE_WAVEFRONT_FP32, args.profile_spp or args.spp, 1)
    pr = ds.render_device(prof_cfg, acc.data_ptr(), acc_w.data_ptr(), profile=True)
    total_stage = sum(pr.stage_ms)
    share = {k: round(v / total_stage, 4) for k, v in zip(("extend", "shade", "shadow", "regen"), pr.stage_ms)}
    # algorithmic bytes of the closest-hit traversal: BVH2 interior nodes (64 B, both child
    # boxes), precomputed-edge triangles (48 B), sphere records (16 B loaded),
    # instance boxes (32 B) + per traced ray: queue index (4 B), ray (32 B), hit (16 B).
    # Camera rays of culled pixels count in rays_closest but are never traced.
    traced = max(pr.rays_closest - pr.sky_samples, 1)
    ext_bytes = (pr.nodes_visited[0] * 64 + pr.tris_tested[0] * 48 + pr.spheres_tested[0] * 16
                 + pr.instances_tested[0] * 32 + traced * (4 + 32 + 16))
    ext_launches = max(pr.stage_launches[0], 1)
    ext_ms = pr.stage_ms[0]
    achieved = ext_bytes / (ext_ms / 1000.0) / 1e9
    peak, peak_kind = measured_peaks()
    per_ray_dram = ncu_traffic_per_ray()
    traffic = per_ray_dram * traced / ext_launches if per_ray_dram else None
    l2_gbs = probe_bandwidth(64 << 20, 50)
    avg_s = ext_ms / ext_launches / 1000.0
    out["roofline"] = {
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
        "traffic": traffic, "kernel": "k_trace<closest> (closest-hit BVH2 traversal)", "peak_kind": peak_kind,
        "traffic_kind": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per traced ray of a saturated "
                         "reduced-case launch (profiles/k_trace_closest_mesh_env_1080p.json) x traced rays per launch here"),
        "algorithmic_bytes_per_launch": ext_bytes / ext_launches, "avg_launch_ms": ext_ms / ext_launches,
        # the resource that binds: the node and triangle reads are served by L1/L2
        "l2_peak": l2_gbs, "l2_peak_kind": "measured live: tpt_probe_read_bandwidth, 64 MiB L2-resident, L1 bypassed",
        "l2_frac": achieved / l2_gbs if l2_gbs else None,
        "dram_frac": (traffic / avg_s / 1e9) / peak if traffic else None,
        "lanes_active": pr.nodes_visited[0] / (32.0 * max(pr.node_steps[0], 1)),
        "lanes_active_shadow": pr.nodes_visited[1] / (32.0 * max(pr.node_steps[1], 1)),
        "lanes_active_scope": "node loop of the traversal: nodes visited / (32 x warp-wide node-loop steps)",
        "lanes_active_leaf": pr.leaf_visits[0] / (32.0 * max(pr.leaf_steps[0], 1)),
        "lanes_active_fast_path": pr.camera_fast / (32.0 * max(pr.fast_steps, 1)),
        "per_ray": {"nodes": pr.nodes_visited[0] / traced,
                    "tris": pr.tris_tested[0] / traced,
                    "spheres": pr.spheres_tested[0] / traced,
                    "bytes": ext_bytes / traced, "scope": "closest-hit rays traced (culled camera rays excluded)"},
        "per_shadow_ray": {"nodes": pr.nodes_visited[1] / max(pr.rays_shadow, 1),
                           "tris": pr.tris_tested[1] / max(pr.rays_shadow, 1),
                           "spheres": pr.spheres_tested[1] / max(pr.rays_shadow, 1),
                           "leaf_visits": pr.leaf_visits[1] / max(pr.rays_shadow, 1),
                           "rays": pr.rays_shadow, "stage_ms": pr.stage_ms[2]},
        "camera_fast_share": pr.camera_fast / traced,
        "camera_culled_share": pr.sky_samples / max(pr.rays_closest, 1),
        "stage_share": share, "profile_spp": prof_cfg.spp,
    }

    # ---- mesh BVH build, device vs host (rank 0, N = 1 only)
    if world == 1 and not args.quick and args.bvh_reps > 0:
        out["bvh_build"] = bvh_leg(args, scene)

    # ---- adaptive Cornell frame (rank 0, N = 1 only)
    if world == 1 and not args.quick and args.adaptive_spp > 0:
        out["adaptive"] = adaptive_leg(args)

    # ---- batch workload (rank 0, N = 1 only)
    if world == 1 and not args.quick and args.batch_scenes > 0:
        out["batch"] = batch_leg(args)
        out["batch_small_scenes"] = small_batch_leg()

    # ---- adjoint ms/step (rank 0, N = 1 only)
    if world == 1 and not args.quick and args.adjoint_steps > 0:
        out["adjoint"] = adjoint_leg(args)

    # ---- CPU baseline (rank 0, N = 1 only)
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, desc, _ = cpu_sample(args, scene, args.cpu_seconds, threads)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc,
                               "cpu": cpu_model()}
        if not args.quick and not args.no_cpu_configs:
            out["cpu_baselines_other_configs"] = cpu_config_baselines(threads)
    out["clocks"] = clocks.summary()
    ds.close()
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.adjoint_only:
        print(json.dumps({"adjoint": adjoint_leg(args)}), flush=True)
        return
    if args.batch_only:
        print(json.dumps({"batch": batch_leg(args), "batch_small_scenes": small_batch_leg()}), flush=True)
        return
    if args.adaptive_only:
        print(json.dumps({"adaptive": adaptive_leg(args)}), flush=True)
        return
    if args.frame_only:
        frame_only(args)
        return
    if args.bvh_only:
        import torch

        torch.cuda.set_device(local_rank)
        print(json.dumps({"bvh_build": bvh_leg(args, build_workload(args))}), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
