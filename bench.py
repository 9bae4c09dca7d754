"""Benchmark of the exact ellipsoid tracer: forward + backward Mrays/s.

Default workload: 1M clustered ellipsoids (SH degree 3), one 1920x1080 view, forward
+ backward through torch.autograd (trace_rays, BVH rebuilt inside every step as the
reference rebuilds its GAS per call). One step = one view traced forward and backward.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). Multi-GPU (torchrun): each rank traces its own view of
the shared scene (weak scaling) and the per-ellipsoid gradients are summed with one
NCCL all-reduce per step. `--impl reference` times the CPU restatement of the
reference's tracer (the reference's OptiX path cannot be built here) on a bounded ray
sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s fwd & fwd+bwd at 1M ellipsoids 1080p; learned-sched vs plain speedup"
UNIT = "Mrays/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--prims", type=int, default=1_000_000)
    p.add_argument("--width", type=int, default=1920)
    p.add_argument("--height", type=int, default=1080)
    p.add_argument("--cpu-sample", type=int, default=0, help="rays in the CPU baseline sample (0: auto)")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--kbuf", type=int, default=0)
    p.add_argument("--block", type=int, default=0)
    p.add_argument("--verbose", action="store_true", help="per-step device times on stderr")
    p.add_argument("--once", action="store_true",
                   help="one scene build + ray order + forward + backward and exit (for ncu captures)")
    return p.parse_args()


def workload(args, rank=0):
    from ever_b200 import synthetic as S
    sc = S.clustered_scene(args.prims, 3, seed=2)
    cam = S.Camera(S.sphere_point(4.0, 2 + rank), args.width, args.height, 50.0)
    ro, rd = S.look_at_rays(cam)
    return sc, ro, rd


def workload_name(args):
    return (f"{args.prims} clustered ellipsoids SH3, {args.width}x{args.height} rays, "
            f"forward+backward via torch.autograd (BVH build per step)")


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.rows = []
        self.proc = None
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            self.sel = uuid if uuid.startswith("GPU-") else f"GPU-{uuid}"
        except Exception:
            self.sel = str(device_index)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.sel, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for n, v in zip(names, r[4:8]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline(sc, ro, rd, threads, target_s=10.0, n_rays=0):
    """The oracle (C++ exact tracer, brute force over all ellipsoids): forward + FP64
    backward on a seeded ray sample sized to about target_s seconds of CPU work."""
    from oracle import oracle as O
    s = O.Scene(sc.mean, sc.scale, sc.quat, sc.density.reshape(-1), sc.features)
    rng = np.random.default_rng(0)
    perm = rng.permutation(ro.shape[0])

    def run(n):
        idx = np.sort(perm[:n])
        o, d = ro[idx], rd[idx]
        t0 = time.perf_counter()
        tr = O.trace(s, o, d, 0.0, 1000.0, 500, nthreads=threads)
        O.backward(s, o, d, 0.0, 1000.0, 500, tr.events, tr.iters, np.ones((n, 5)), nthreads=threads)
        return time.perf_counter() - t0

    if not n_rays:
        n0 = max(2 * threads, 8)
        dt0 = run(n0)
        n_rays = int(min(ro.shape[0], max(n0, target_s / max(dt0 / n0, 1e-9))))
    dt = run(n_rays)
    return n_rays / dt / 1e6, dt, n_rays


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sc, ro, rd = workload(args)
    threads = os.cpu_count() or 1
    _, _, n = cpu_baseline(sc, ro, rd, threads, target_s=4.0, n_rays=args.cpu_sample)
    vals = []
    for i in range(args.warmup + args.steps):
        v, dt, _ = cpu_baseline(sc, ro, rd, threads, n_rays=n)
        if i >= args.warmup:
            vals.append(v)
    value = float(np.median(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * ro.shape[0] / (value * 1e6),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded clustered scene; no trained scenes ship with the reference)",
        "config": {"workload": workload_name(args), "sample": f"{n} seeded rays of the view per step"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n} rays of the {args.width}x{args.height} view per step, all ellipsoids"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference OptiX/Slang tracer unavailable on this box (no OptiX SDK, slangc, glm, CGAL, absl); "
                "timed: the CPU restatement of its trace path (oracle/ever_oracle.cpp)",
    }
    print(json.dumps(line), flush=True)


def run_once(args):
    """One untimed pass of the hot path through the tracer API: what an ncu capture profiles."""
    import torch
    from ever_b200 import tracer as T
    dev = torch.device("cuda", 0)
    sc, ro, rd = workload(args)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=dev)
    rayo, rayd = t(ro), t(rd)
    tune = T.Tune(kbuf=args.kbuf or 16, block=args.block or 128)
    scene = T.Scene(t(sc.mean), t(sc.scale), t(sc.quat), t(sc.density.reshape(-1)), t(sc.features))
    order = T.ray_order(rayo, rayd)
    fwd = T.forward(scene, rayo, rayd, 0.0, 1000.0, 500, ray_order=order, tune=tune)
    T.backward(scene, rayo, rayd, fwd, torch.ones((rayo.shape[0], 5), device=dev), 0.0, 1000.0, 500,
               ray_order=order, tune=tune)
    torch.cuda.synchronize()
    print(json.dumps({"once": True, "rays": int(rayo.shape[0]), "status": int(fwd.status.item()),
                      "events_per_ray": float(fwd.iters.float().mean().item())}))


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.once:
        return run_once(args)
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    from ever_b200 import distributed as D
    from ever_b200 import tracer as T
    from ever_b200.fast_ellipsoid_splinetracer import trace_rays

    sc, ro, rd = workload(args, rank)
    R = ro.shape[0]
    tune = None
    if args.kbuf or args.block:
        tune = T.Tune(kbuf=args.kbuf or 16, block=args.block or 128)
    host = {k: np.ascontiguousarray(v.reshape(v.shape[0], -1) if k == "density" else v) for k, v in
            dict(mean=sc.mean, scale=sc.scale, quat=sc.quat, density=sc.density, features=sc.features).items()}
    params = {k: torch.tensor(v, device=dev, requires_grad=True) for k, v in host.items()}
    rayo = torch.tensor(ro, device=dev)
    rayd = torch.tensor(rd, device=dev)
    gout = torch.randn((R, 5), generator=torch.Generator().manual_seed(rank), dtype=torch.float32).to(dev)

    def step():
        for p in params.values():
            p.grad = None
        out = trace_rays(params["mean"], params["scale"], params["quat"], params["density"], params["features"],
                         rayo, rayd, 0.0, 1000.0, 3, None, None, 500, False, None, tune)
        out.backward(gout)
        if world > 1:
            D.allreduce_gradients([p.grad for p in params.values()])
        return out

    for i in range(args.warmup):
        if args.verbose:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            step()
            b.record()
            torch.cuda.synchronize()
            print(f"warmup step {i}: {a.elapsed_time(b):.2f} ms", file=sys.stderr, flush=True)
        else:
            step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record()
        marks = []
        for _ in range(args.steps):
            step()
            if args.verbose:
                marks.append(torch.cuda.Event(enable_timing=True))
                marks[-1].record()
        ev1.record()
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    if args.verbose:
        prev = ev0
        for i, m in enumerate(marks):
            print(f"timed step {i}: {prev.elapsed_time(m):.2f} ms", file=sys.stderr, flush=True)
            prev = m
    ms = D.max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dev)
    value = world * R / (ms * 1e-3) / 1e6

    # ---- phase breakdown (outside the timed region): build / forward / backward kernels
    def phases(reps=3):
        scene_t = [params[k].detach() for k in ("mean", "scale", "quat", "density", "features")]
        res = {"order": [], "build": [], "fwd": [], "bwd": []}
        for _ in range(reps):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
            e[0].record()
            order = T.ray_order(rayo, rayd)
            e[1].record()
            scene = T.Scene(*scene_t)
            e[2].record()
            fwd = T.forward(scene, rayo, rayd, 0.0, 1000.0, 500, tune=tune, ray_stats=True, ray_order=order)
            e[3].record()
            T.backward(scene, rayo, rayd, fwd, gout, 0.0, 1000.0, 500, tune=tune, ray_order=order)
            e[4].record()
            torch.cuda.synchronize()
            res["order"].append(e[0].elapsed_time(e[1]))
            res["build"].append(e[1].elapsed_time(e[2]))
            res["fwd"].append(e[2].elapsed_time(e[3]))
            res["bwd"].append(e[3].elapsed_time(e[4]))
        med = {k: float(np.median(v)) for k, v in res.items()}
        stats = fwd.ray_stats
        med["events_per_ray"] = float(stats[:, 0].mean().item())
        return med

    ph = phases()

    # ---- end to end through the public API with host buffers (pinned), per step:
    # H2D of the ellipsoids and rays, trace_rays forward + backward, D2H of the image
    pinned = {k: torch.from_numpy(v).pin_memory() for k, v in host.items()}
    ro_h, rd_h = torch.from_numpy(ro).pin_memory(), torch.from_numpy(rd).pin_memory()
    out_h = torch.empty((R, 5), dtype=torch.float32).pin_memory()
    h2d = sum(v.numel() * 4 for v in pinned.values()) + ro_h.numel() * 4 + rd_h.numel() * 4
    d2h = out_h.numel() * 4

    def e2e_step():
        p = {k: v.to(dev, non_blocking=True).requires_grad_(True) for k, v in pinned.items()}
        o = ro_h.to(dev, non_blocking=True)
        d = rd_h.to(dev, non_blocking=True)
        out = trace_rays(p["mean"], p["scale"], p["quat"], p["density"], p["features"], o, d, 0.0, 1000.0, 3,
                         None, None, 500, False, None, tune)
        out.backward(gout)
        out_h.copy_(out.detach(), non_blocking=True)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        e2e_step()
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = D.max_over_ranks(e0.elapsed_time(e1) / args.steps, dev)
    e2e_value = world * R / (e2e_ms * 1e-3) / 1e6

    # ---- roofline of the dominant kernel (algorithmic bytes per launch / launch time)
    N = args.prims
    P = 12 + 12 + 16 + 4 + 12 * 16
    b_fwd = N * P + R * (24 + 20) + R * (64 + 4)
    b_bwd = 2 * N * P + R * (24 + 20 + 68 + 24)
    peak, peak_kind = measured_peaks()
    dom = "bwd" if ph["bwd"] >= ph["fwd"] else "fwd"
    b_dom = b_bwd if dom == "bwd" else b_fwd
    achieved = b_dom / (ph[dom] * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": "k_trace_bwd" if dom == "bwd" else "k_trace_fwd",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": None,
                "algorithmic_bytes": b_dom}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded clustered scene; no trained scenes ship with the reference)",
        "config": {"workload": workload_name(args), "global_batch": world * R, "rays_per_gpu": R,
                   "ellipsoids": N, "sh_degree": 3, "max_iters": 500,
                   "parallelism": f"rays sharded by view, dp{world}",
                   "l2": "inputs larger than L2 (scene 236 MB + rays 50 MB per step)"},
        "fwd_mrays_trace_only": R / (ph["fwd"] * 1e-3) / 1e6,
        "fwd_mrays_with_build": R / ((ph["fwd"] + ph["build"] + ph["order"]) * 1e-3) / 1e6,
        "fwdbwd_mrays_trace_only": R / ((ph["fwd"] + ph["bwd"]) * 1e-3) / 1e6,
        "fwdbwd_mrays_with_build": R / ((ph["fwd"] + ph["bwd"] + ph["build"] + ph["order"]) * 1e-3) / 1e6,
        "phase_ms": ph,
        "clocks": clk.summary(),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": args.steps * 20,
        "roofline": roofline,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        v, dt, n = cpu_baseline(sc, ro, rd, threads, target_s=10.0, n_rays=args.cpu_sample)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{n} seeded rays of the view, forward + FP64 backward, {dt:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
