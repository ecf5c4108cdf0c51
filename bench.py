#!/usr/bin/env python
"""Benchmark of the LLG time-stepping hot path on B200.

Workload (default): the plain FP32 method on a single 3D grid of
256 x 256 x 32 cells of 4 x 4 x 4 nm, Ms = 1.1e6 A/m, Aex = 1.5e-11 J/m,
uniaxial Ku = 5e5 J/m^3 along z, alpha = 0.5, m = independent unit vectors
uniform on the sphere (seed 2), zero field, Heun with a fixed dt = 1e-14 s.
A step is one Heun step (two effective-field evaluations) of the whole grid.

Prints one JSON line (rank 0).  Metric: cell-steps/s, whole job.
  --impl ours       the fused B200 engine (mmx_* C ABI)
  --impl reference  the reference's path on the host cores: MuMax 1 has no
                    CPU implementation, so this is the CPU restatement of its
                    algorithm (oracle/, FP32, OpenMP over all host threads)
Multi-GPU: one process per GPU, each advancing its own replica of the grid
(the single-grid path does not shard); value = all ranks' cell-steps / the
slowest rank's time.
"""
import argparse
import ctypes
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "plain-fp32-heun-256x256x32": dict(
        grid=(256, 256, 32), cell=(4e-9, 4e-9, 4e-9), msat=1.1e6, aexch=1.5e-11, alpha=0.5, anis=1, k1=5e5,
        axis=(0, 0, 1), solver="heun", dt=1e-14, seed=2, init="random"),
    "plain-fp32-heun-128x32x1": dict(
        grid=(128, 32, 1), cell=(3.90625e-9, 3.90625e-9, 3e-9), msat=8.0e5, aexch=1.3e-11, alpha=0.02,
        bext=(-24.6e-3, 4.3e-3, 0.0), solver="heun", dt=1e-14, seed=1, init="tilted"),
}
BATCH_WORKLOADS = {
    # batching workload: 256 uneven instances (seed 4), RK4, fixed dt 5e-15 s
    "batch-fp32-rk4-256": dict(count=256, seed=4, solver="rk4", dt=5e-15),
}
SERVE_WORKLOADS = {
    # serving workload: Poisson stream of 200 req/s, seed 5, relaxations
    # (alpha 1, stop at max torque < 1e-4) and 21-point sweeps of B along x
    # from -100 to +100 mT; a bounded sample of the stream's first requests.
    # dt None: each request's stable RK4 step (1_b200.stable_dt)
    "serve-fp32-rk4-mixed": dict(seed=5, rate=200.0, dt=None, max_torque=1e-4, check_every=100, points=21),
}
ADAPTIVE_WORKLOADS = {
    # 128 x 32 x 1 thin film (standard-problem-4 geometry), RK23, max error 1e-5
    "plain-fp32-rk23-128x32x1": dict(
        grid=(128, 32, 1), cell=(3.90625e-9, 3.90625e-9, 3e-9), msat=8.0e5, aexch=1.3e-11, alpha=0.02,
        bext=(-24.6e-3, 4.3e-3, 0.0), solver="rk23", maxerror=1e-5, seed=1, init="tilted"),
}
PRECISION_WORKLOADS = {
    # precision workload: 512 x 512 x 1 film of 2 nm cells,
    # Ms 8.6e5, A 1.3e-11, alpha 0.1, vortex-like m (seed 3), RK23 1e-5
    "precision-bf16x3-rk23-512x512": dict(
        grid=(512, 512, 1), cell=(2e-9, 2e-9, 2e-9), msat=8.6e5, aexch=1.3e-11, alpha=0.1, solver="rk23",
        maxerror=1e-5, seed=3),
}
DEFAULT = "plain-fp32-heun-256x256x32"


def sim_kwargs(w):
    keys = ("grid", "cell", "msat", "aexch", "alpha", "bext", "anis", "k1", "axis", "solver", "dt")
    return {k: w[k] for k in keys if k in w}


def seeded_m(grid, seed, mode):
    """Internal [3][X][Y][Z] magnetisation: user components (x,y,z) drawn as
    default_rng(seed).standard_normal((3, nz, ny, nx)); internal component C
    is user component 2-C."""
    nx, ny, nz = grid
    u = np.random.default_rng(seed).standard_normal((3, nz, ny, nx))
    v = 1.0 + 0.01 * u if mode == "tilted" else u
    v = v / np.sqrt((v * v).sum(axis=0, keepdims=True))
    return np.ascontiguousarray(v[::-1]).astype(np.float32)


def pass_bytes(w):
    """Algorithmic HBM bytes per launch of each kernel of one field
    evaluation of the zero-aware padded convolution, and per cell-step for
    Heun (two evaluations plus the predictor/corrector state).

    3D: zfwd (read m, write Z spectra of the data rows), yfwd, xconv (X
    transform + kernel multiply + inverse, reads the kernel octant), yinv,
    zinv_epi (read Z spectra, Heun state in/out).  2D: zfwd, yconv2d,
    zinv_epi."""
    nx, ny, nz = w["grid"]
    N0, N1, N2 = nz, ny, nx
    P0 = 2 * N0 if N0 > 1 else 1
    P1, P2 = 2 * N1, 2 * N2
    HZ = P2 // 2 + 1
    n = N0 * N1 * N2
    zspec = 3 * N0 * N1 * HZ * 8      # Z-transformed data rows
    yspec = 3 * N0 * P1 * HZ * 8      # after the Y transform
    heun_epi = (36 + 48) * n // 2     # mean of predictor and corrector state traffic
    if P0 > 1:
        koct = 6 * (P0 // 2 + 1) * (P1 // 2 + 1) * HZ * 4
        b = {"zfwd": 3 * n * 4 + zspec, "yfwd": zspec + yspec, "xconv": 2 * yspec + koct,
             "yinv": yspec + zspec, "zinv_epi": zspec + heun_epi}
    else:
        koct = 4 * (P1 // 2 + 1) * HZ * 4
        b = {"zfwd": 3 * n * 4 + zspec, "yconv2d": 2 * zspec + koct, "zinv_epi": zspec + heun_epi}
    per_step = 2 * sum(b.values())  # the model's bytes per Heun step (separate passes)
    # the fused pass of a fixed-step Heun run (inverse Z + epilogue + the next
    # forward Z): the spectrum rows in and out, the Heun state, m not re-read
    b["zinv_epi_zfwd"] = 2 * zspec + heun_epi
    state = 9 * n * 4 + (yspec if P0 > 1 else zspec) + koct
    return b, per_step / n, state


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a run."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                       "-lms", "100", "-i", str(device)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.f.read().splitlines():
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel, workload):
    """Per-launch DRAM bytes of 'kernel' from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get(workload, {}).get(kernel)


def cpu_baseline(w, steps_budget_s=20.0):
    """The CPU restatement of the reference's algorithm (oracle, FP32,
    OpenMP over all host threads) on the same workload: bounded sample of
    whole-grid steps after one untimed step."""
    import oracle as O
    kw = sim_kwargs(w)
    cfg = O.make_cfg(**kw)
    m = seeded_m(w["grid"], w["seed"], w["init"])
    t0 = time.perf_counter()
    o = O.OracleSim(cfg, m, bits=32)
    setup = time.perf_counter() - t0
    o.steps(1)
    n = int(np.prod(w["grid"]))
    done, t0 = 0, time.perf_counter()
    while True:
        o.steps(1)
        done += 1
        el = time.perf_counter() - t0
        if el > steps_budget_s or done >= 50:
            break
    return {"value": n * done / el, "unit": "cell-steps/s", "cores": O.num_threads(), "kind": "port",
            "steps_timed": done,
            "sample": "%d whole-grid Heun steps of %s after 1 untimed step (setup incl. kernel %.1f s untimed)" % (
                done, "x".join(map(str, w["grid"])), setup)}


def run_batch(args, name):
    """The batched form: many uneven-size instances, one launch per pass and
    line length, one CUDA graph per step."""
    import torch
    eng = importlib.import_module("1_b200")
    bw = BATCH_WORKLOADS[name]
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    cfgs = eng.batch_config(bw["count"], seed=bw["seed"], solver=bw["solver"], dt=bw["dt"])
    t0 = time.perf_counter()
    b = eng.Batch([eng.mmx_params(**c) for c in cfgs])
    setup = time.perf_counter() - t0
    for i, (inst, c) in enumerate(zip(b.instances, cfgs)):
        inst.set_m(seeded_m(c["grid"], 1000 + i, "random"))
        inst.normalize()
    info = b.size()
    stream = torch.cuda.Stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    b.use_graph(True)
    b.step(args.warmup, sh)
    torch.cuda.synchronize()
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(args.steps, sh)
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    cells = info["cells"]
    line = {"metric": "cell-steps/s", "value": cells * args.steps / (ms / 1e3), "unit": "cell-steps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": name, "instances": info["count"], "cells": cells, "solver": bw["solver"],
                       "dt_s": bw["dt"], "launches_per_step": info["launches_per_step"],
                       "setup_s": setup},
            "instance_steps_per_s": info["count"] * args.steps / (ms / 1e3),
            "gpu_launches": info["launches_per_step"] * args.steps, "clocks": clk}
    b.close()
    print(json.dumps(line), flush=True)


def pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(np.ceil(q / 100.0 * len(xs))) - 1))
    return xs[k]


def run_serve(args, name):
    """The serving form: the request loop with continuous batching against
    the same loop solving one request at a time (the plain form), on the
    same requests with the same arrival times.  Requests of the stream are
    partitioned over the ranks (no collective on the data path)."""
    import torch
    eng = importlib.import_module("1_b200")
    sw = SERVE_WORKLOADS[name]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    reqs = eng.serve_stream(args.requests, seed=sw["seed"], rate=sw["rate"], dt=sw["dt"], sweep_points=sw["points"])
    part = eng.partition_requests(reqs, world)
    mine = [r for r, k in zip(reqs, part) if k == rank]
    out = {}
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    arms = ["served", "plain"] if not args.no_plain else ["served"]
    for arm in arms:
        sv = eng.Server(batched=(arm == "served"), check_every=sw["check_every"], keep_m=True)
        t0 = time.perf_counter()
        res = eng.run_stream(sv, mine, realtime=True, max_torque=sw["max_torque"], max_steps=args.serve_max_steps)
        wall = time.perf_counter() - t0
        ms = {r["index"]: sv.result_m(r["id"]) for r in res}
        st = sv.stats()
        sv.close()
        lat = [r["latency"] for r in res]
        out[arm] = dict(res=res, m=ms, wall=wall, stats=st,
                        solves_per_s=len(res) / wall if wall > 0 else 0.0,
                        p50_ms=1e3 * pct(lat, 50), p99_ms=1e3 * pct(lat, 99),
                        steps=sum(r["steps"] for r in res),
                        converged=sum(1 for r in res if r["converged"]))
    clk = clocks.stop()
    same = None
    if "plain" in out:
        same = max(float(np.abs(out["served"]["m"][i] - out["plain"]["m"][i]).max()) for i in out["served"]["m"])
    srv = out["served"]
    cells = {r["index"]: int(np.prod(r["cfg"]["grid"])) for r in mine}
    cell_steps = sum(cells[r["index"]] * r["steps"] for r in srv["res"])
    line = {"metric": "solves/s", "value": srv["solves_per_s"], "unit": "solves/s", "n_gpus": world,
            "steps": len(mine), "warmup": 0, "ms_per_step": 1e3 * srv["wall"] / max(1, len(mine)),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": name, "requests": len(mine), "stream_requests": len(reqs),
                       "rate_per_s": sw["rate"], "seed": sw["seed"], "dt_s": sw["dt"] or "stable_dt per request",
                       "max_torque": sw["max_torque"], "check_every": sw["check_every"],
                       "sweep_points": sw["points"], "max_steps_per_point": args.serve_max_steps,
                       "sample": "the first %d requests of the stream, arriving in real time" % len(reqs)},
            "latency_ms": {"p50": srv["p50_ms"], "p99": srv["p99_ms"]},
            "served": {"solves_per_s": srv["solves_per_s"], "wall_s": srv["wall"], "steps": srv["steps"],
                       "cell_steps_per_s": cell_steps / srv["wall"], "converged": srv["converged"],
                       "chunks": srv["stats"]["chunks"], "regroups": srv["stats"]["regroups"]},
            "clocks": clk}
    if "plain" in out:
        pl = out["plain"]
        line["plain"] = {"solves_per_s": pl["solves_per_s"], "wall_s": pl["wall"], "p50_ms": pl["p50_ms"],
                         "p99_ms": pl["p99_ms"], "steps": pl["steps"]}
        line["speedup_vs_plain"] = srv["solves_per_s"] / pl["solves_per_s"] if pl["solves_per_s"] else None
        line["served_vs_plain_max_abs_dm"] = same
    line["per_request"] = [{"i": r["index"], "kind": r["kind"], "grid": list(next(q["cfg"]["grid"] for q in mine
                                                                               if q["index"] == r["index"])),
                            "steps": r["steps"], "latency_ms": 1e3 * r["latency"], "converged": r["converged"]}
                           for r in srv["res"]]
    by_kind = {}
    for r in srv["res"]:
        by_kind.setdefault(r["kind"], []).append(r)
    line["served"]["by_kind"] = {k: {"requests": len(v), "converged": sum(1 for r in v if r["converged"]),
                                     "p50_ms": 1e3 * pct([r["latency"] for r in v], 50),
                                     "p99_ms": 1e3 * pct([r["latency"] for r in v], 99),
                                     "steps": sum(r["steps"] for r in v)} for k, v in sorted(by_kind.items())}
    if world > 1:
        import torch.distributed as dist
        lines = [None] * world
        dist.gather_object(line, lines if rank == 0 else None, dst=0)
        if rank == 0:
            tot = sum(len(l["per_request"]) for l in lines)
            wall = max(l["served"]["wall_s"] for l in lines)
            lat = [q["latency_ms"] for l in lines for q in l["per_request"]]
            line["value"] = tot / wall
            line["latency_ms"] = {"p50": pct(lat, 50), "p99": pct(lat, 99)}
            line["config"]["requests"] = tot
    if rank == 0:
        print(json.dumps(line), flush=True)


def vortex_m(nx, ny, seed=3, core=2.5, noise=0.02):
    """In-plane curl about the film centre, +z within `core` cells of it,
    plus noise * N(0,1) per component (default_rng(seed)), normalised;
    internal layout [3][1][ny][nx] (internal component C = user 2-C)."""
    y, x = np.mgrid[0:ny, 0:nx].astype(np.float64)
    x -= (nx - 1) / 2.0
    y -= (ny - 1) / 2.0
    r = np.hypot(x, y)
    u = np.zeros((3, 1, ny, nx))
    u[0, 0] = -y / np.maximum(r, 1e-12)
    u[1, 0] = x / np.maximum(r, 1e-12)
    inner = r <= core
    u[0, 0][inner] = 0.0
    u[1, 0][inner] = 0.0
    u[2, 0][inner] = 1.0
    u += noise * np.random.default_rng(seed).standard_normal(u.shape)
    u /= np.sqrt((u * u).sum(axis=0, keepdims=True))
    return np.ascontiguousarray(u[::-1]).astype(np.float32)


def run_precision(args, name):
    """The precision form against the FP32 form on the same film: RK23
    steps per second of each, the split-precision field's difference from
    the FP32 form's (one evaluation) and the two forms' difference after the
    same number of steps.  Their error against FP64 is a test
    (tests/test_gpu_precision.py)."""
    import torch
    eng = importlib.import_module("1_b200")
    w = PRECISION_WORKLOADS[name]
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    nx, ny, _ = w["grid"]
    n = nx * ny
    m0 = vortex_m(nx, ny, w["seed"])
    kw = {k: w[k] for k in ("grid", "cell", "msat", "aexch", "alpha", "solver", "maxerror")}
    stream = torch.cuda.Stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    res = {}
    for prec in (1, 0):
        s = eng.Solver(eng.mmx_params(**kw, precision=prec))
        s.set_m(m0, sh)
        s.normalize(sh)
        s.step(args.warmup, sh)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step(args.steps, sh)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        st = s.state()
        # per-pass times
        s.profile(True)
        s.step(min(args.steps, 50), sh)
        torch.cuda.synchronize()
        times = s.pass_times()
        s.profile(False)
        res[prec] = dict(ms=ms, state=st, m=s.get_m(), passes={k: v[0] / v[1] for k, v in times.items()})
        # field of the initial state for the FP64 comparison
        mt = torch.from_numpy(m0).cuda()
        ht = torch.zeros_like(mt)
        s.field(ctypes.c_void_p(mt.data_ptr()), ctypes.c_void_p(ht.data_ptr()))
        torch.cuda.synchronize()
        res[prec]["h"] = ht.cpu().numpy()
        s.close()
    clk = clocks.stop()
    p, f = res[1], res[0]
    scale = float(np.abs(f["h"]).max())
    value = n * args.steps / (p["ms"] / 1e3)
    line = {"metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": p["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3 split, f32 accumulate", "data": "synthetic",
            "config": {"workload": name, "grid": list(w["grid"]), "solver": "rk23", "maxerror": w["maxerror"],
                       "init": "vortex, seed 3"},
            "fp32_form": {"value": n * args.steps / (f["ms"] / 1e3), "ms_per_step": f["ms"] / args.steps,
                          "passes_ms_per_launch": f["passes"]},
            "passes_ms_per_launch": p["passes"],
            "field_diff_vs_fp32_form": {"split_bf16": float(np.abs(p["h"] - f["h"]).max()) / scale,
                                        "norm": "max |h_split - h_fp32| / max |h_fp32|, one evaluation of the "
                                                "initial state; the error against FP64 is measured by "
                                                "tests/test_gpu_precision.py"},
            "gpu_launches": None, "clocks": clk}
    # same number of adaptive steps: compare the states where both forms stand
    line["after_steps"] = {"steps": args.warmup + args.steps, "time_split": p["state"]["time"],
                           "time_fp32": f["state"]["time"],
                           "max_abs_dm_split_vs_fp32": float(np.abs(p["m"] - f["m"]).max())}
    print(json.dumps(line), flush=True)


def run_adaptive(args, name):
    """RK23 on the small film: accepted steps per second with the host dt
    controller (8 bytes read back per trial, as the reference's two
    reductions per step) and with the device controller (graph-replayed
    trials, one read-back at the end)."""
    import torch
    eng = importlib.import_module("1_b200")
    w = ADAPTIVE_WORKLOADS[name]
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = int(np.prod(w["grid"]))
    m0 = seeded_m(w["grid"], w["seed"], w["init"])
    kw = {k: w[k] for k in ("grid", "cell", "msat", "aexch", "alpha", "bext", "solver", "maxerror")}
    stream = torch.cuda.Stream()
    sh = ctypes.c_void_p(stream.cuda_stream)
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    out = {}
    for mode in ("device", "host"):
        s = eng.Solver(eng.mmx_params(**kw))
        s.set_m(m0, sh)
        s.normalize(sh)
        if mode == "device":
            s.device_control(True)
        s.step(args.warmup, sh)
        st0 = s.state()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step(args.steps, sh)
        e1.record(stream)
        e1.synchronize()
        wall = time.perf_counter() - t0
        st1 = s.state()
        acc = st1["steps"] - st0["steps"]
        out[mode] = dict(ms=e0.elapsed_time(e1), wall=wall, accepted=acc, sim_time=st1["time"] - st0["time"],
                         calls=args.steps)
        s.close()
    clk = clocks.stop()
    d, h = out["device"], out["host"]
    value = n * d["accepted"] / (d["ms"] / 1e3)
    line = {"metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": 1,
            "steps": d["accepted"], "warmup": args.warmup, "ms_per_step": d["ms"] / max(1, d["accepted"]),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": name, "grid": list(w["grid"]), "solver": "rk23", "maxerror": w["maxerror"],
                       "controller": "device (graph per trial)"},
            "device_controller": {"trials": d["calls"], "accepted": d["accepted"],
                                  "accepted_steps_per_s": d["accepted"] / (d["ms"] / 1e3)},
            "host_controller": {"accepted": h["accepted"], "accepted_steps_per_s": h["accepted"] / (h["ms"] / 1e3),
                                "value": n * h["accepted"] / (h["ms"] / 1e3)},
            "clocks": clk}
    print(json.dumps(line), flush=True)


def kernel_host(eng, torch, params):
    """The real-space demag + exchange kernel of the padded grid, built on
    the GPU (mmx_face_kernel6), as the host array the driver restatement
    takes."""
    N = tuple(params.size)
    per = tuple(params.periodic)
    Pd = tuple(2 * n if (n > 1 and p == 0) else n for n, p in zip(N, per))
    out = torch.zeros((6,) + Pd, device="cuda")
    eng.face_kernel6_device(Pd, per, [params.cellsize[d] for d in range(3)], exch6=True,
                            out_ptr=ctypes.c_void_p(out.data_ptr()))
    torch.cuda.synchronize()
    k = out.cpu().numpy()
    del out
    return k


def time_driver(eng, torch, w, m0, libpath, steps=20, warmup=2):
    """Whole-grid steps per second of a libgpukern implementation driven by
    the Go-driver restatement (libmmxdriver.so).  The reference's library
    synchronises the device after every primitive; this library's
    primitives return once queued on the default stream.  The wall clock
    runs from a device synchronisation to one after the last step, so it is
    the device time plus the launch gaps the call sequence imposes."""
    kw = sim_kwargs(w)
    k6 = kernel_host(eng, torch, eng.mmx_params(**kw))
    d = eng.DriverSim(eng.driver_config(**kw), m0, k6, libpath=libpath)
    d.steps(warmup)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    d.steps(steps)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    d.close()
    n = int(np.prod(w["grid"]))
    return {"value": n * steps / el, "unit": "cell-steps/s", "ms_per_step": 1e3 * el / steps, "steps": steps,
            "warmup": warmup, "library": os.path.relpath(libpath, ROOT),
            "path": "Go-driver restatement (libmmxdriver.so) over the libgpukern C ABI, the call sequence of the "
                    "unchanged Go front end"}


def run_reference(args, w, name):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cb = cpu_baseline(w)
    # a bounded sample: the whole-grid steps actually timed, not --steps
    line = {"metric": "cell-steps/s", "value": cb["value"], "unit": "cell-steps/s", "n_gpus": 1,
            "steps": cb["steps_timed"], "warmup": 1, "steps_requested": args.steps,
            "warmup_requested": args.warmup, "ms_per_step": 1e3 * np.prod(w["grid"]) / cb["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": name, "grid": list(w["grid"]), "solver": w["solver"], "dt_s": w["dt"],
                       "parallelism": "host threads (rank 0)"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    # context: the reference's own CUDA library (cuFFT, synchronous
    # primitives), built from its sources for sm_100a, driven by the
    # Go-driver restatement on the same workload
    ref_lib = os.path.join(ROOT, "oracle", "_ref", "libgpukern_ref.so")
    if args.no_reference_gpu:
        pass
    elif not os.path.exists(ref_lib):
        line["reference_gpu"] = {"unavailable": "oracle/_ref/libgpukern_ref.so was not built"}
    else:
        try:
            import torch
            if torch.cuda.is_available():
                eng = importlib.import_module("1_b200")
                m0 = seeded_m(w["grid"], w["seed"], w["init"])
                line["reference_gpu"] = time_driver(eng, torch, w, m0, ref_lib, steps=args.drop_in_steps)
            else:
                line["reference_gpu"] = {"unavailable": "no CUDA device"}
        except Exception as e:  # context only: never fail the CPU arm
            line["reference_gpu"] = {"unavailable": "%s: %s" % (type(e).__name__, e)}
    print(json.dumps(line), flush=True)


def run_ours(args, w, name):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    eng = importlib.import_module("1_b200")
    kw = sim_kwargs(w)
    n = int(np.prod(w["grid"]))
    m0 = seeded_m(w["grid"], w["seed"], w["init"])
    s = eng.Solver(eng.mmx_params(**kw))
    stream = torch.cuda.Stream()
    sh = ctypes.c_void_p(stream.cuda_stream)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    # ---- device-resident timed region (graph replay per step) ----
    s.set_m(m0, sh)
    s.normalize(sh)
    s.use_graph(True)
    s.step(args.warmup, sh)
    barrier()
    clocks = Clocks(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    s.step(args.steps, sh)
    ev1.record(stream)
    ev1.synchronize()
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    t = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    value = world * n * args.steps / (ms / 1e3)

    # ---- per-kernel durations: event-record nodes inside the step graph ----
    s.profile(2)
    ksteps = min(args.steps, 200)
    s.step(ksteps, sh)
    torch.cuda.synchronize()
    times = s.pass_times()
    s.profile(False)
    barrier()

    # ---- the drop-in path: this library's primitives under the Go-driver
    # restatement (the call sequence the unchanged Go front end issues) ----
    drop_in = None
    if world == 1 and not args.no_drop_in:
        drop_in = time_driver(eng, torch, w, m0, eng.LIB_PATH, steps=args.drop_in_steps)

    # ---- end to end through the C ABI with host buffers ----
    s.use_graph(True)
    pin_in = torch.from_numpy(m0.reshape(-1)).pin_memory()
    pin_out = torch.empty(3 * n, dtype=torch.float32).pin_memory()
    pin_avg = torch.empty((args.steps, 3), dtype=torch.float32).pin_memory()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    eng.lib().mmx_solver_set_m(s.h, ctypes.c_void_p(pin_in.data_ptr()), 1, sh)
    s.normalize(sh)
    row = pin_avg.data_ptr()
    for k in range(args.steps):
        s.step(1, sh)
        s.avg_m(ctypes.c_void_p(row + 12 * k), True, sh)
    eng.lib().mmx_solver_get_m(s.h, ctypes.c_void_p(pin_out.data_ptr()), 1, sh)
    e1.record(stream)
    e1.synchronize()
    barrier()
    ems = e0.elapsed_time(e1)
    t = torch.tensor([ems], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ems = float(t.item())
    e2e = world * n * args.steps / (ems / 1e3)
    avg_last = pin_avg[-1].tolist()
    s.close()
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return

    b, bytes_per_cell_step, state = pass_bytes(w)
    peak, peak_kind = measured_peaks()
    dom = max(times, key=lambda k: times[k][0])
    # each event node between two passes adds a gap of its own (the next
    # kernel cannot start before the event is recorded): the event-timed
    # step exceeds the step timed without event nodes (the timed region
    # above) by that gap per pass, which is taken off every pass equally
    ev_step_ms = sum(v[0] for v in times.values()) / ksteps
    passes_per_step = launches_per_step = sum(la for _, la in times.values()) / ksteps
    gap_ms = max(0.0, (ev_step_ms - ms / args.steps) / passes_per_step) if passes_per_step else 0.0
    per_launch = {k: v[0] / v[1] - gap_ms for k, v in times.items()}
    dom_ms = per_launch[dom]
    achieved = b[dom] / (dom_ms / 1e3) / 1e9
    traffic = ncu_traffic(dom, name)
    line = {
        "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": name, "grid": list(w["grid"]), "cell_m": list(w["cell"]), "solver": w["solver"],
                   "dt_s": w["dt"], "parallelism": "replicas x%d" % world,
                   "l2": "working set %.0f MB per GPU vs 126 MB L2 (no flush between steps)" % (state / 1e6)},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": b[dom], "avg_launch_ms": dom_ms,
                     "step_bytes_per_cell": bytes_per_cell_step,
                     "step_frac": bytes_per_cell_step * value / world / 1e9 / peak,
                     "passes_ms_per_launch": per_launch,
                     "passes_timing": "event-record nodes between the passes inside the step graph (%d steps): "
                                      "the event-timed step (%.4f ms) exceeds the %.4f ms step timed without "
                                      "event nodes by %.4f ms per pass, taken off each pass" %
                                      (ksteps, ev_step_ms, ms / args.steps, gap_ms),
                     "passes_ms_per_launch_events": {k: v[0] / v[1] for k, v in times.items()}},
        "e2e": {"value": e2e, "unit": "cell-steps/s",
                "h2d_bytes_per_step": 3 * n * 4 / args.steps,
                "d2h_bytes_per_step": 12 + 3 * n * 4 / args.steps,
                "path": "mmx C ABI: m from pinned host, per-step <m> to pinned host, final m to host",
                "avg_m_last": avg_last},
        "gpu_launches": int(round(launches_per_step * args.steps)),
        "clocks": clk,
    }
    if drop_in is not None:
        line["drop_in"] = drop_in
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT,
                    choices=sorted(WORKLOADS) + sorted(BATCH_WORKLOADS) + sorted(SERVE_WORKLOADS) +
                    sorted(PRECISION_WORKLOADS) + sorted(ADAPTIVE_WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--requests", type=int, default=16, help="serving: requests of the stream to run")
    ap.add_argument("--serve-max-steps", type=int, default=0, help="serving: step cap per relaxation (0: none)")
    ap.add_argument("--no-plain", action="store_true", help="serving: skip the one-at-a-time arm")
    ap.add_argument("--no-drop-in", action="store_true", help="skip timing the drop-in primitive path")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip timing the reference's own CUDA library")
    ap.add_argument("--drop-in-steps", type=int, default=20)
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: start the ranks here when not under torchrun
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
               "--master-addr", "127.0.0.1", "--master-port", str(29500 + os.getpid() % 1000)] + sys.argv
        sys.exit(subprocess.call(cmd))
    if args.workload in SERVE_WORKLOADS:
        if int(os.environ.get("WORLD_SIZE", "1")) > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo", init_method="env://")
        run_serve(args, args.workload)
        return
    if args.workload in ADAPTIVE_WORKLOADS:
        run_adaptive(args, args.workload)
        return
    if args.workload in PRECISION_WORKLOADS:
        run_precision(args, args.workload)
        return
    if args.workload in BATCH_WORKLOADS:
        run_batch(args, args.workload)
        return
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, w, args.workload)
    else:
        run_ours(args, w, args.workload)


if __name__ == "__main__":
    main()
