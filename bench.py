#!/usr/bin/env python
"""Benchmark of the batched spline hot path (build + evaluate) on B200.

Workload (default): the non-uniform quintic configuration -- degree-5 B-splines on 1024 cells with
break points = uniform grid + U[-0.3h, 0.3h] noise, Hermite closures (derivative orders 1 and 2 at
each end), 65536 batch lines in the (x, batch) layout, built from cos(2 pi k x + phi) samples and
differentiated (first derivative) at 1024 random points per line. FP64 arithmetic.

One step = one SplineBuilder call over all lines + one SplineEvaluator::deriv call over all lines.
metric: Gpts/s = (lines * interpolation points + lines * evaluation points) / 2 / step time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one rank per GPU (the script starts torchrun itself when it is not already under it):
the global batch is N x 65536 lines and every rank builds and evaluates its own contiguous shard of
it (weak scaling, no collective on the data path); time = max over ranks of the CUDA-event time.
`--cpu-stub` runs the same rank logic (launch, sharding, timing, max over ranks) on CPU ranks over
gloo with a small NumPy step in place of the GPU kernels, for testing the multi-rank plumbing.
`--impl reference` times the reference algorithm's CPU restatement (oracle/, the reference's
schedule: host factorisation, thread-per-line sweeps, OpenMP over lines) on a bounded sample.
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

METRIC = "spline build+eval Gpts/s & %HBM peak; FP64 vs FP32+refine at <=1e-12 rel err"
UNIT = "Gpts/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--lines", type=int, default=1 << 16, help="batch lines per GPU")
    p.add_argument("--e2e-steps", type=int, default=0, help="steps of the host-buffer (e2e) timing; 0 = --steps")
    p.add_argument("--e2e-slice", type=int, default=4096, help="lines per slice of the host pipeline (e2e)")
    p.add_argument("--cpu-seconds", type=float, default=10.0, help="target CPU time of the baseline sample")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--tile-lines", type=int, default=0, help="builder tile width (0 = plan default)")
    p.add_argument("--chunks", type=int, default=0, help="builder chunks per line (0 = plan default)")
    p.add_argument("--no-configs", action="store_true", help="skip the other configurations' measurements")
    p.add_argument("--cpu-stub", action="store_true",
                   help="CPU ranks (gloo) with a NumPy step in place of the GPU kernels: checks the rank logic only")
    p.add_argument("--profile-case", choices=["adjoint", "periodic_cubic", "tensor2d", "uneven", "quintic", "quintic_refine"], default=None,
                   help="run only this case's kernels, --steps times on --lines lines (for profilers; prints no JSON line)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload_plan(D, lines):
    from ddc_b200 import workloads

    br = workloads.config2_breaks(1024)
    bs = D.NonUniformBSplines(5, False, br)
    pts = D.greville_points(bs, D.SplineBuilderClosure.HERMITE, D.SplineBuilderClosure.HERMITE)
    return bs, pts, br


def make_inputs(pts, lines, m, line0=0, total=None):
    """Inputs of lines [line0, line0 + lines) of a batch of `total` lines."""
    from ddc_b200 import workloads

    return workloads.config2(B=lines, points=pts, m=m, line0=line0, total=total)


class Ranks:
    """One process per GPU (or per CPU rank under --cpu-stub): rank / world from the torchrun
    environment, the process group, this rank's shard of the global batch and the max over ranks."""

    def __init__(self, backend, device=None):
        import torch.distributed as dist

        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = dist if self.world > 1 else None
        if self.dist is not None:
            from datetime import timedelta

            kw = {"device_id": device} if device is not None else {}
            dist.init_process_group(backend, timeout=timedelta(seconds=120), **kw)

    def shard(self, lines_per_rank):
        """[start, stop) of this rank's lines in the global batch of world * lines_per_rank lines."""
        from ddc_b200.sharding import shard_range

        return shard_range(self.world * lines_per_rank, self.rank, self.world)

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, value, device=None):
        """Max of a float over ranks (every rank takes part)."""
        if self.dist is None:
            return float(value)
        import torch

        t = torch.tensor([float(value)], dtype=torch.float64, device=device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def gather(self, obj):
        if self.dist is None:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()


def run_cpu_stub(args):
    """The multi-rank logic of run_ours on CPU ranks (gloo): each rank draws its shard of the global
    batch, times a NumPy stand-in for the kernels (the sum of its samples times its coordinates)
    over `steps` steps after `warmup`, and rank 0 prints the JSON line with the max over ranks.
    Only the plumbing is under test here; no number it prints is a measurement of the path."""
    R = Ranks("gloo")
    lines, m = args.lines, 64
    start, stop = R.shard(lines)
    pts = np.linspace(0.0, 1.0, 33)
    w = make_inputs(pts, stop - start, m, line0=start, total=R.world * lines)
    step = lambda: float(w["vals"].sum() + w["coords"].sum())
    for _ in range(args.warmup):
        step()
    R.barrier()
    t0 = time.perf_counter()
    check = 0.0
    for _ in range(args.steps):
        check = step()
    ms = (time.perf_counter() - t0) * 1e3
    ms_max = R.max(ms)
    shards = R.gather([start, stop, check])
    if R.rank == 0:
        total = R.world * lines * (pts.size + m) / 2
        print(json.dumps({"impl": "cpu-stub", "metric": METRIC, "value": total / (ms_max / args.steps * 1e-3) / 1e9,
                          "unit": UNIT, "n_gpus": R.world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": ms_max / args.steps, "scaling": "weak",
                          "config": {"lines_per_gpu": lines, "global_lines": R.world * lines,
                                     "parallelism": f"batch-sharded x{R.world}"},
                          "shards": shards}), flush=True)
    R.close()


def relaunch_under_torchrun(args):
    """--gpus N > 1 outside torchrun: start N ranks (this script under torchrun, 127.0.0.1) and
    return their exit status; rank 0 prints the JSON line."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def algorithmic_bytes(lines, npts, nder, ncoef, m):
    build = lines * (npts + nder) * 8 + lines * ncoef * 8
    ev = lines * ncoef * 8 + lines * m * 8 * 2
    return build, ev


def cpu_reference_rate(lines_sample, seconds, threads=None):
    """Time the oracle (reference schedule) on `lines_sample` lines: build + first-derivative eval."""
    from oracle import oracle as O
    from ddc_b200 import workloads

    br = workloads.config2_breaks(1024)
    obs = O.BSplines(5, False, breaks=br)
    pts = obs.greville(O.HERMITE, O.HERMITE)
    ob = O.Builder(obs, pts, O.HERMITE, O.HERMITE)
    w = workloads.config2(B=lines_sample, points=pts, m=1024)
    nt = threads or O.max_threads()
    reps, t_total = 0, 0.0
    t0 = time.perf_counter()
    while True:
        t1 = time.perf_counter()
        c = ob(w["vals"], w["dlo"], w["dhi"], nthreads=nt)
        O.evaluate(obs, w["coords"], c, order=1, nthreads=nt)
        t_total += time.perf_counter() - t1
        reps += 1
        if time.perf_counter() - t0 > seconds:
            break
    pts_per_rep = lines_sample * (pts.size + 1024) / 2
    return pts_per_rep * reps / t_total / 1e9, nt, reps, t_total


def workload_config(lines, m, world):
    """The `config` of both arms' JSON lines: the workload the metric is quoted on."""
    return {"workload": "non-uniform quintic Hermite B-splines, 1024 cells (1025 points + 2x2 derivatives), "
                        f"{lines} lines per GPU in (x, batch) layout, build + first derivative at {m} random points "
                        "per line",
            "lines_per_gpu": lines, "degree": 5, "ncells": 1024, "eval_points_per_line": m,
            "l2": "inputs larger than L2 (2.2 GB touched per step)", "parallelism": f"batch-sharded x{world}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # each step is a bounded sample of the workload: 512 lines (of 65536) built and differentiated
    from oracle import oracle as O

    O.lib()
    sample = 512
    rates = []
    for i in range(args.warmup + args.steps):
        r, nt, reps, tt = cpu_reference_rate(sample, 0.0)
        if i >= args.warmup:
            rates.append(r)
    value = float(np.median(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {**workload_config(args.lines, 1024, args.gpus), "sample_lines_per_step": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nt, "kind": "port",
                         "sample": f"{sample} lines per step (build + first-derivative eval), oracle/ restatement "
                                   "of the reference's LAPACK path with its thread-per-line OpenMP schedule"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _converged(builder):
    """Whether the refined solves queued so far met the builder's bound (ddcb_builder_device_status)."""
    try:
        builder.device_status()
        return True
    except Exception:
        return False


def _time_ms(fn, reps, rotate=1):
    """Mean CUDA-event time of fn(i) over `reps` calls after 3 warm-ups; i cycles over `rotate`
    buffer sets (several sets larger than L2 in all keep each call's inputs out of L2)."""
    import torch

    for i in range(3):
        fn(i % rotate)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(reps):
        fn(i % rotate)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def measure_configs(peak, reps):
    """The other configurations of the path, each at its named size (FP64 I/O, synthetic inputs):
    periodic cubic 1000x1000 (build + evaluate), non-uniform quintic Hermite in FP32 + refinement,
    the 2D periodic x Hermite cubic 512^2 x 64 fields, the uneven batch of 4096 problems, and the
    differentiation step (forward and adjoint) on periodic cubic, 1024 cells x 65536 lines."""
    import torch

    import ddc_b200 as D
    from ddc_b200 import workloads as W

    dev = torch.device("cuda")
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    out = {}
    # ---- periodic uniform cubic, 1000 cells x 1000 lines, build + evaluate at 1000 points/line ----
    w = W.config1()
    bs = D.UniformBSplines(3, True, 0.0, 1.0, 1000)
    b, e = D.SplineBuilder(bs), D.SplineEvaluator(bs)
    sets = 8  # 8 x 40 MB > 2 x L2
    vals = [cu(w["vals"]) for _ in range(sets)]
    xs = [cu(w["coords"]) for _ in range(sets)]
    cs = [torch.empty((bs.size, 1000), dtype=torch.float64, device=dev) for _ in range(sets)]
    ys = [torch.empty((1000, 1000), dtype=torch.float64, device=dev) for _ in range(sets)]
    fused = b.build_and_evaluate(e, cs[0], vals[0], xs[0], ys[0])
    step = lambda i: b.build_and_evaluate(e, cs[i], vals[i], xs[i], ys[i])
    ms_rot = _time_ms(step, 10 * reps, sets)
    ms_l2 = _time_ms(step, 10 * reps, 1)
    pts = 1000 * (1000 + 1000) / 2
    bytes_fused = 1000 * 1000 * 8 + 1000 * 1003 * 8 + 1000 * 1000 * 16
    # the same with a builder planned for 128 chunks per line (the chunks option): a batch this
    # small gives each SM one 8-line tile, whose 1024 threads all sweep with 128 chunks
    b128 = D.SplineBuilder(bs, chunks=128)
    step128 = lambda i: b128.build_and_evaluate(e, cs[i], vals[i], xs[i], ys[i])
    ms128 = _time_ms(step128, 10 * reps, sets)
    out["periodic_cubic_1000x1000"] = {
        "schedule": "fused build+eval kernel" if fused else "two kernels",
        "ms": ms_rot, "Gpts_per_s": pts / ms_rot / 1e6, "GBps": bytes_fused / ms_rot / 1e6,
        "hbm_frac": bytes_fused / ms_rot / 1e6 / peak, "ms_l2_resident": ms_l2,
        "chunks_128": {"ms": ms128, "GBps": bytes_fused / ms128 / 1e6, "hbm_frac": bytes_fused / ms128 / 1e6 / peak},
        "note": "8 rotating buffer sets (320 MB) for the HBM figure; one set for the L2-resident one; "
                "default builder options, and chunks_128 with the builder option chunks=128"}
    del vals, xs, cs, ys
    # ---- non-uniform quintic Hermite, 65536 lines: FP64 vs FP32 + FP64 refinement -------------
    br = W.config2_breaks(1024)
    bs = D.NonUniformBSplines(5, False, br)
    pts2 = D.greville_points(bs, 1, 1)
    w = W.config2(B=1 << 16, points=pts2)
    v, lo, hi = cu(w["vals"]), cu(w["dlo"]), cu(w["dhi"])
    ref = torch.empty((bs.size, 1 << 16), dtype=torch.float64, device=dev)
    b64 = D.SplineBuilder(bs, pts2, 1, 1)
    t64 = _time_ms(lambda i: b64(ref, v, lo, hi), reps)
    prec = {"fp64_build_ms": t64}
    for rounds in (1, 2):
        br_ = D.SplineBuilder(bs, pts2, 1, 1, precision="fp32_refine", refine_rounds=rounds)
        c = torch.empty_like(ref)
        t = _time_ms(lambda i: br_(c, v, lo, hi), reps)
        err = float((c - ref).abs().max() / ref.abs().max())
        prec[f"fp32_refine_{rounds}_rounds"] = {"build_ms": t, "speedup_vs_fp64": t64 / t, "max_rel_err_vs_fp64": err,
                                                "converged": _converged(br_)}
    out["quintic_hermite_precision"] = prec
    # ---- the same lines integrated straight from the samples (build + integrate in one pass) ----
    integ = torch.empty(1 << 16, dtype=torch.float64, device=dev)
    ti = _time_ms(lambda i: b64.integrate_samples(integ, v, lo, hi), 10 * reps)
    ib = (v.numel() + lo.numel() + hi.numel() + integ.numel()) * 8
    out["quintic_hermite_integrate_samples"] = {"ms": ti, "GBps": ib / ti / 1e6, "hbm_frac": ib / ti / 1e6 / peak}
    del v, lo, hi, ref, integ
    # ---- 2D: periodic cubic x Hermite cubic, 512 x 512, 64 fields ------------------------------
    w = W.config3()
    bx, by = D.UniformBSplines(3, True, 0.0, 1.0, 512), D.UniformBSplines(3, False, 0.0, 1.0, 512)
    Bx, By = D.SplineBuilder(bx, None, 0, 0), D.SplineBuilder(by, None, 1, 1)
    b2, e2 = D.SplineBuilder2D(Bx, By), D.SplineEvaluator2D(D.SplineEvaluator(bx), D.SplineEvaluator(by))
    v, d0, d1, x = cu(w["vals"]), cu(w["dmin2"]), cu(w["dmax2"]), cu(w["coords"])
    c2 = torch.empty((bx.size, by.size, 64), dtype=torch.float64, device=dev)
    y2 = torch.empty(v.shape, dtype=torch.float64, device=dev)
    # a caller that repeats the build keeps its workspace (no stream-ordered allocation per call)
    ws2 = torch.empty(b2.workspace_bytes(64) // 8 + 1, dtype=torch.float64, device=dev)
    tb = _time_ms(lambda i: b2(c2, v, derivs_min2=d0, derivs_max2=d1, workspace=ws2), reps)
    te = _time_ms(lambda i: e2(y2, x, c2), reps)
    n2 = v.numel()
    b_bytes = (n2 + d0.numel() + d1.numel() + c2.numel()) * 8
    e_bytes = (c2.numel() + 3 * n2) * 8
    out["tensor2d_512x512x64"] = {"build_ms": tb, "eval_ms": te, "Gpts_per_s": n2 / (tb + te) / 1e6,
                                  "build_GBps": b_bytes / tb / 1e6, "eval_GBps": e_bytes / te / 1e6,
                                  "hbm_frac": (b_bytes + e_bytes) / (tb + te) / 1e6 / peak}
    # FP32 + refinement (the named precision of this configuration), error against the FP64 build
    Bxr = D.SplineBuilder(bx, None, 0, 0, precision="fp32_refine", refine_rounds=1)
    Byr = D.SplineBuilder(by, None, 1, 1, precision="fp32_refine", refine_rounds=1)
    b2r = D.SplineBuilder2D(Bxr, Byr)
    c2r = torch.empty_like(c2)
    tbr = _time_ms(lambda i: b2r(c2r, v, derivs_min2=d0, derivs_max2=d1, workspace=ws2), reps)
    out["tensor2d_512x512x64"]["fp32_refine_1_round"] = {
        "build_ms": tbr, "speedup_vs_fp64": tb / tbr, "max_rel_err_vs_fp64": float((c2r - c2).abs().max() / c2.abs().max()),
        "converged": _converged(Bxr) and _converged(Byr)}
    # the x-advection of the step (velocity per y row, feet computed in the fused kernel)
    vy = cu(w["v"])
    ya = torch.empty_like(v)
    ex = D.SplineEvaluator(bx)
    fused_adv = Bx.advect(ex, ya, v, w["dt"], vy, velocity_div=64)
    ta = _time_ms(lambda i: Bx.advect(ex, ya, v, w["dt"], vy, velocity_div=64), reps)
    ab = 2 * v.numel() * 8
    out["advection_x_512x512x64"] = {"ms": ta, "GBps": ab / ta / 1e6, "hbm_frac": ab / ta / 1e6 / peak,
                                     "schedule": "fused kernel, feet computed in it" if fused_adv else "three kernels"}
    del v, d0, d1, x, c2, y2, ws2, c2r, ya
    # ---- uneven batch: 4096 problems, FP32 + refinement (its named precision) -------------------
    probs = W.config4()
    wr = W.config4_batch(D, probs, precision="fp32_refine", refine_rounds=2)
    batch = D.UnevenBatch(wr["builders"], wr["evaluators"], wr["nevals"])
    rinfo = batch.info
    rv, rlo, rhi, rx = cu(wr["vals"]), cu(wr["dlo"]), cu(wr["dhi"]), cu(wr["coords"])
    rc = torch.empty((rinfo.total_coefs,), dtype=torch.float64, device=dev)
    ry = torch.empty((rinfo.total_evals,), dtype=torch.float64, device=dev)
    rtinf = batch.tune(rv, rlo, rhi, rc, rx, ry, reps=3)
    trefine = _time_ms(lambda i: batch(rv, rlo, rhi, rc, rx, ry), 10 * reps)
    r_conv = all(_converged(b) for b in wr["builders"])
    del batch, rv, rlo, rhi, rx
    # ---- uneven batch: 4096 problems, FP64 ----------------------------------------------------
    wb = W.config4_batch(D, probs)
    batch = D.UnevenBatch(wb["builders"], wb["evaluators"], wb["nevals"])
    info = batch.info
    bv, blo, bhi, bx_ = cu(wb["vals"]), cu(wb["dlo"]), cu(wb["dhi"]), cu(wb["coords"])
    bc = torch.empty((info.total_coefs,), dtype=torch.float64, device=dev)
    by_ = torch.empty((info.total_evals,), dtype=torch.float64, device=dev)
    tinf = batch.tune(bv, blo, bhi, bc, bx_, by_, reps=3)
    tbatch = _time_ms(lambda i: batch(bv, blo, bhi, bc, bx_, by_), 10 * reps)
    off = batch.offsets()
    views = []
    for i, (bb, ee) in enumerate(zip(wb["builders"], wb["evaluators"])):
        sl = lambda t, k: t[off[k][i]:off[k][i + 1]][:, None]
        views.append((bb, ee, sl(bv, "vals"), sl(blo, "derivs_lo") if off["derivs_lo"][i + 1] > off["derivs_lo"][i] else None,
                      sl(bhi, "derivs_hi") if off["derivs_hi"][i + 1] > off["derivs_hi"][i] else None,
                      sl(bc, "coefs"), sl(bx_, "evals"), sl(by_, "evals")))

    def loop(i):
        for bb, ee, vv, ll, hh, cc, xx, yy in views:
            bb(cc, vv, ll, hh)
            ee(yy, xx, cc)

    tloop = _time_ms(loop, 2)
    r_err = float((rc - bc).abs().max() / bc.abs().max())
    ub = 8 * (info.total_vals + info.total_derivs_lo + info.total_derivs_hi + info.total_coefs + 2 * info.total_evals)
    out["uneven_batch_4096"] = {"problems": int(info.count), "points": int(info.total_vals), "evals": int(info.total_evals),
                                "ms": tbatch, "Gpts_per_s": (info.total_vals + info.total_evals) / 2 / tbatch / 1e6,
                                "GBps": ub / tbatch / 1e6, "loop_per_problem_fp64_ms": tloop, "speedup_vs_loop": tloop / tbatch,
                                "schedule": {"warp_schedule": bool(tinf.warp_schedule), "threads": tinf.threads,
                                             "budget_256_threads_per_sm": tinf.blocks_per_sm,
                                             "order": "largest-first" if tinf.order == 0 else "natural"},
                                "fp32_refine_2_rounds": {"ms": trefine, "Gpts_per_s": (info.total_vals + info.total_evals) / 2 / trefine / 1e6,
                                                        "max_rel_err_vs_fp64_coefs": r_err, "converged": r_conv,
                                                        "warp_schedule": bool(rtinf.warp_schedule)}}
    del batch, wb, views, bv, blo, bhi, bx_, bc, by_
    # ---- differentiation: periodic cubic 1024 cells, 65536 lines, 1024 points/line ------------
    B, m = 1 << 16, 1024
    bs = D.UniformBSplines(3, True, 0.0, 1.0, 1024)
    b, e = D.SplineBuilder(bs), D.SplineEvaluator(bs)
    gen = torch.Generator(device=dev).manual_seed(5)
    x = torch.rand((m, B), dtype=torch.float64, device=dev, generator=gen)
    g = torch.randn((m, B), dtype=torch.float64, device=dev, generator=gen)
    v = torch.randn((1024, B), dtype=torch.float64, device=dev, generator=gen)
    c = torch.empty((1027, B), dtype=torch.float64, device=dev)
    y = torch.empty((m, B), dtype=torch.float64, device=dev)
    gv = torch.empty((1024, B), dtype=torch.float64, device=dev)
    gx = torch.empty((m, B), dtype=torch.float64, device=dev)
    tf = _time_ms(lambda i: b.build_and_evaluate(e, c, v, x, y), reps)
    tb_ = _time_ms(lambda i: b.build_and_evaluate_adjoint(e, x, c, g, gv, gx), reps)
    fwd_bytes = B * (1024 + 1027 + 2 * m) * 8
    bwd_bytes = B * (m + m + 1027 + m + 1024) * 8
    out["adjoint_periodic_cubic_1024x65536"] = {"fwd_ms": tf, "bwd_ms": tb_, "fwd_GBps": fwd_bytes / tf / 1e6,
                                                "bwd_GBps": bwd_bytes / tb_ / 1e6, "bwd_hbm_frac": bwd_bytes / tb_ / 1e6 / peak}
    # the forward in FP32 + refinement (this configuration's named precision)
    br5 = D.SplineBuilder(bs, precision="fp32_refine", refine_rounds=1)
    c5, y5 = torch.empty_like(c), torch.empty_like(y)
    tf5 = _time_ms(lambda i: br5.build_and_evaluate(e, c5, v, x, y5), reps)
    b.build_and_evaluate(e, c, v, x, y)
    out["adjoint_periodic_cubic_1024x65536"]["fwd_fp32_refine_1_round"] = {
        "ms": tf5, "speedup_vs_fp64": tf / tf5, "max_rel_err_vs_fp64_values": float((y5 - y).abs().max() / y.abs().max()),
        "converged": _converged(br5)}
    del x, g, v, c, y, gv, gx, c5, y5
    # ---- the advection step of periodic cubic 1000 cells x 1000 lines (feet in the kernel) ----
    bs1 = D.UniformBSplines(3, True, 0.0, 1.0, 1000)
    b1, e1 = D.SplineBuilder(bs1), D.SplineEvaluator(bs1)
    sets = 8
    f_in = [torch.randn((1000, 1000), dtype=torch.float64, device=dev) for _ in range(sets)]
    f_out = [torch.empty((1000, 1000), dtype=torch.float64, device=dev) for _ in range(sets)]
    fused1 = b1.advect(e1, f_out[0], f_in[0], 0.37e-3, 1.0)
    ta1 = _time_ms(lambda i: b1.advect(e1, f_out[i], f_in[i], 0.37e-3, 1.0), 10 * reps, sets)
    ab1 = 2 * 1000 * 1000 * 8
    out["advection_periodic_cubic_1000x1000"] = {"ms": ta1, "GBps": ab1 / ta1 / 1e6, "hbm_frac": ab1 / ta1 / 1e6 / peak,
                                                 "schedule": "fused kernel, feet computed in it" if fused1 else "three kernels",
                                                 "note": "8 rotating buffer sets (128 MB)"}
    del f_in, f_out
    # ---- 3D: periodic cubic x Hermite cubic x Greville cubic, 96^3 cells, 16 fields ----------
    n3, F = 96, 16
    b3 = [D.UniformBSplines(3, True, 0.0, 1.0, n3), D.UniformBSplines(3, False, 0.0, 1.0, n3),
          D.UniformBSplines(3, False, 0.0, 1.0, n3)]
    B3 = [D.SplineBuilder(b3[0]), D.SplineBuilder(b3[1], None, 1, 1), D.SplineBuilder(b3[2], None, 3, 3)]
    bld3 = D.SplineBuilder3D(*B3)
    np3 = [bb.npoints for bb in B3]
    v3 = torch.randn((np3[0], np3[1], np3[2], F), dtype=torch.float64, device=dev)
    dm = torch.randn((np3[0], 1, np3[2], F), dtype=torch.float64, device=dev)
    dM = torch.randn((np3[0], 1, np3[2], F), dtype=torch.float64, device=dev)
    c3 = torch.empty((b3[0].size, b3[1].size, b3[2].size, F), dtype=torch.float64, device=dev)
    ws3 = torch.empty(bld3.workspace_bytes(F) // 8 + 1, dtype=torch.float64, device=dev)
    tb3 = _time_ms(lambda i: bld3(c3, v3, workspace=ws3, derivs_min2=dm, derivs_max2=dM), reps)
    ev3 = D.SplineEvaluator3D(*[D.SplineEvaluator(bb) for bb in b3])
    # evaluation points shared by the fields (as the feet of an advection step are)
    x3 = torch.rand((np3[0] * np3[1] * np3[2] // 4, 1, 3), dtype=torch.float64, device=dev).expand(-1, F, 3).contiguous()
    y3 = torch.empty((x3.shape[0], F), dtype=torch.float64, device=dev)
    te3 = _time_ms(lambda i: ev3(y3, x3, c3), reps)
    bb3 = (v3.numel() + dm.numel() + dM.numel() + c3.numel()) * 8
    eb3 = (c3.numel() + x3.numel() + y3.numel()) * 8
    out["tensor3d_96cubed_x16"] = {"build_ms": tb3, "eval_ms": te3, "build_GBps": bb3 / tb3 / 1e6,
                                   "eval_points": int(y3.numel()), "eval_Gpts_per_s": y3.numel() / te3 / 1e6,
                                   "eval_GBps_algorithmic": eb3 / te3 / 1e6}
    return out


def run_ours(args):
    import torch

    import ddc_b200 as D

    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available() or local >= torch.cuda.device_count():
        raise RuntimeError(f"rank {local} has no CUDA device (found {torch.cuda.device_count()})")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    R = Ranks("nccl", dev)
    world, rank = R.world, R.rank
    # this rank's shard of the global batch (world x --lines lines); no collective on the data path
    start, stop = R.shard(args.lines)
    lines, m = stop - start, 1024
    bs, pts, br = workload_plan(D, lines)
    builder = D.SplineBuilder(bs, pts, D.SplineBuilderClosure.HERMITE, D.SplineBuilderClosure.HERMITE,
                              tile_lines=args.tile_lines, chunks=args.chunks)
    ev = D.SplineEvaluator(bs)
    w = make_inputs(pts, lines, m, line0=start, total=world * args.lines)
    h_vals = torch.from_numpy(w["vals"]).pin_memory()
    h_dlo = torch.from_numpy(w["dlo"]).pin_memory()
    h_dhi = torch.from_numpy(w["dhi"]).pin_memory()
    h_x = torch.from_numpy(w["coords"]).pin_memory()
    vals, dlo, dhi, x = (t.to(dev) for t in (h_vals, h_dlo, h_dhi, h_x))
    coefs = torch.empty((bs.size, lines), dtype=torch.float64, device=dev)
    out = torch.empty((m, lines), dtype=torch.float64, device=dev)
    h_out = torch.empty((m, lines), dtype=torch.float64).pin_memory()
    s = torch.cuda.current_stream()

    def step_fused():
        builder.build_and_evaluate(ev, coefs, vals, x, out, dlo, dhi, order=1)

    def step_two_calls():
        builder(coefs, vals, dlo, dhi)
        ev.deriv(1, out, x, coefs)

    for _ in range(args.warmup):
        step_fused()
        step_two_calls()
    torch.cuda.synchronize()
    R.barrier()
    fused = builder.build_and_evaluate(ev, coefs, vals, x, out, dlo, dhi, order=1)
    # ---- device-resident timing of the fused step (inputs > L2: 2.2 GB touched per step) ----
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    R.barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(s)
    for i in range(args.steps):
        evs[i][0].record(s)
        step_fused()
        evs[i][1].record(s)
    t1.record(s)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = t0.elapsed_time(t1)
    f_ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
    # ---- the two-call schedule (SplineBuilder then SplineEvaluator::deriv), per kernel ----
    ev_b = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    ev_e = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        ev_b[i][0].record(s)
        builder(coefs, vals, dlo, dhi)
        ev_b[i][1].record(s)
        ev_e[i][0].record(s)
        ev.deriv(1, out, x, coefs)
        ev_e[i][1].record(s)
    torch.cuda.synchronize()
    b_ms = float(np.mean([a.elapsed_time(b) for a, b in ev_b]))
    e_ms = float(np.mean([a.elapsed_time(b) for a, b in ev_e]))
    ms = R.max(ms, dev)
    ms_step = ms / args.steps
    npts = pts.size
    total_pts = world * lines * (npts + m) / 2
    value = total_pts / (ms_step * 1e-3) / 1e9
    # ---- end-to-end through the public API with host buffers: the host pipeline
    # (ddcb_host_pipeline_run) copies every step's inputs in and its result out, batch slices
    # overlapping the kernels ----
    ke = args.e2e_steps or args.steps
    pipe = D.HostPipeline(builder, ev, m, order=1, slice_lines=args.e2e_slice)
    for _ in range(2):
        pipe(h_vals, h_x, h_out, h_dlo, h_dhi, stream=s)
    torch.cuda.synchronize()
    R.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(ke):
        pipe(h_vals, h_x, h_out, h_dlo, h_dhi, stream=s)
    e1.record(s)
    torch.cuda.synchronize()
    e_ms_total = e0.elapsed_time(e1)
    e_ms_total = R.max(e_ms_total, dev)
    e2e_value = total_pts / (e_ms_total / ke * 1e-3) / 1e9
    e2e_matches = bool(torch.equal(h_out, out.cpu()))  # the device-resident step ran on the same inputs
    h2d = sum(t.numel() * 8 for t in (h_vals, h_dlo, h_dhi, h_x))
    d2h = h_out.numel() * 8
    # ---- roofline of the dominant kernel: the fused build + derivative kernel when the step ran
    # as one kernel, else the longer of the builder and evaluator kernels ----
    b_bytes, e_bytes = algorithmic_bytes(lines, npts, 4, bs.size, m)
    f_bytes = b_bytes + lines * m * 16  # coefficients written once, never re-read
    peak, peak_kind = peaks()
    if fused:
        kname, kbytes, kms, kkey = "build_eval_kernel (fused build + deriv)", f_bytes, f_ms, "build_eval_kernel"
    elif e_ms >= b_ms:
        kname, kbytes, kms, kkey = "eval_kernel (first derivative)", e_bytes, e_ms, "eval_kernel"
    else:
        kname, kbytes, kms, kkey = "build_kernel", b_bytes, b_ms, "build_kernel"
    achieved = kbytes / (kms * 1e-3) / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            traffic = json.load(f).get(kkey)
    except Exception:
        pass
    result = None
    if rank == 0:
        cpu = None
        if not args.no_cpu and world == 1:
            try:
                r, nt, reps, tt = cpu_reference_rate(256, args.cpu_seconds)
                cpu = {"value": r, "unit": UNIT, "cores": nt, "kind": "port",
                       "sample": f"256 of the 65536 lines (build + first-derivative eval at 1024 points), {reps} reps "
                                 f"in {tt:.1f} s, oracle/ restatement of the reference's LAPACK path"}
            except Exception as exc:  # the baseline is reported, not required
                cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "port", "sample": f"failed: {exc}"}
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {**workload_config(lines, m, world),
                       "schedule": "fused build+deriv kernel" if fused else "builder kernel then evaluator kernel"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": kname,
                         "algorithmic_bytes_per_launch": kbytes, "peak_kind": peak_kind},
            "kernels": {"step_ms": f_ms, "step_algorithmic_GBps": (f_bytes if fused else b_bytes + e_bytes) / (f_ms * 1e-3) / 1e9,
                        "per_kernel": {"build_ms": b_ms, "eval_ms": e_ms,
                                     "build_GBps": b_bytes / (b_ms * 1e-3) / 1e9,
                                     "eval_GBps": e_bytes / (e_ms * 1e-3) / 1e9,
                                     "Gpts_per_s": total_pts / ((b_ms + e_ms) * 1e-3) / 1e9 / world}},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": ke, "path": f"ddcb_host_pipeline_run, {args.e2e_slice}-line slices, pinned host buffers",
                    "matches_device_path": e2e_matches},
            "gpu_launches": args.steps if fused else 2 * args.steps,
            "clocks": clk,
        }
        if not args.no_configs and world == 1:
            try:
                result["configs"] = measure_configs(peak, max(3, args.steps // 2))
            except Exception as exc:  # reported, not required for the headline line
                result["configs"] = {"error": f"{type(exc).__name__}: {exc}"}
        print(json.dumps(result), flush=True)
    R.close()
    return result


def profile_case(args):
    """A short run of one case's kernels at a chosen batch, for ncu captures on small workloads:
    adjoint = periodic cubic 1024 cells, build + evaluate then its backward; periodic_cubic = the
    fused build + evaluate of 1000 cells; tensor2d = the 2D build and evaluation of 512 x 512 cells
    over --lines fields; uneven = the 4096-problem uneven batch (untuned schedule); quintic = the
    headline's builder and first-derivative evaluator on --lines lines; quintic_refine = its
    builder in FP32 with one FP64 refinement round."""
    import torch

    import ddc_b200 as D
    from ddc_b200 import workloads as W

    dev = torch.device("cuda")
    B = args.lines
    gen = torch.Generator(device=dev).manual_seed(5)
    if args.profile_case in ("adjoint", "periodic_cubic"):
        n = 1024 if args.profile_case == "adjoint" else 1000
        bs = D.UniformBSplines(3, True, 0.0, 1.0, n)
        b, e = D.SplineBuilder(bs), D.SplineEvaluator(bs)
        x = torch.rand((n, B), dtype=torch.float64, device=dev, generator=gen)
        v = torch.randn((n, B), dtype=torch.float64, device=dev, generator=gen)
        g = torch.randn((n, B), dtype=torch.float64, device=dev, generator=gen)
        c = torch.empty((bs.size, B), dtype=torch.float64, device=dev)
        y = torch.empty((n, B), dtype=torch.float64, device=dev)
        gv, gx = torch.empty_like(v), torch.empty_like(x)
        for _ in range(args.steps):
            b.build_and_evaluate(e, c, v, x, y)
            if args.profile_case == "adjoint":
                b.build_and_evaluate_adjoint(e, x, c, g, gv, gx)
    elif args.profile_case == "uneven":
        probs = W.config4()
        wb = W.config4_batch(D, probs)
        batch = D.UnevenBatch(wb["builders"], wb["evaluators"], wb["nevals"])
        info = batch.info
        cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        bv, blo, bhi, bx = cu(wb["vals"]), cu(wb["dlo"]), cu(wb["dhi"]), cu(wb["coords"])
        bc = torch.empty((info.total_coefs,), dtype=torch.float64, device=dev)
        by = torch.empty((info.total_evals,), dtype=torch.float64, device=dev)
        for _ in range(args.steps):
            batch(bv, blo, bhi, bc, bx, by)
    elif args.profile_case in ("quintic", "quintic_refine"):
        bs, pts, br = workload_plan(D, B)
        prec = "fp32_refine" if args.profile_case == "quintic_refine" else "fp64"
        builder = D.SplineBuilder(bs, pts, D.SplineBuilderClosure.HERMITE, D.SplineBuilderClosure.HERMITE,
                                  precision=prec, refine_rounds=1)
        ev = D.SplineEvaluator(bs)
        w = make_inputs(pts, B, 1024)
        cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        vals, dlo, dhi, x = cu(w["vals"]), cu(w["dlo"]), cu(w["dhi"]), cu(w["coords"])
        coefs = torch.empty((bs.size, B), dtype=torch.float64, device=dev)
        out = torch.empty((1024, B), dtype=torch.float64, device=dev)
        for _ in range(args.steps):
            builder(coefs, vals, dlo, dhi)
            ev.deriv(1, out, x, coefs)
    else:
        w = W.config3(nfields=B)
        cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        bx, by = D.UniformBSplines(3, True, 0.0, 1.0, 512), D.UniformBSplines(3, False, 0.0, 1.0, 512)
        b2 = D.SplineBuilder2D(D.SplineBuilder(bx, None, 0, 0), D.SplineBuilder(by, None, 1, 1))
        e2 = D.SplineEvaluator2D(D.SplineEvaluator(bx), D.SplineEvaluator(by))
        v, d0, d1, x = cu(w["vals"]), cu(w["dmin2"]), cu(w["dmax2"]), cu(w["coords"])
        c2 = torch.empty((bx.size, by.size, B), dtype=torch.float64, device=dev)
        y2 = torch.empty(v.shape, dtype=torch.float64, device=dev)
        for _ in range(args.steps):
            b2(c2, v, derivs_min2=d0, derivs_max2=d1)
            e2(y2, x, c2)
    torch.cuda.synchronize()


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch_under_torchrun(args))
    if args.cpu_stub:
        run_cpu_stub(args)
        return
    if args.profile_case:
        profile_case(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
