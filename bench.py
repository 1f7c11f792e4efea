"""Benchmark: batched BytecodeTape gradient + HVP throughput on B200.

Default workload (the configuration the headline metric is quoted on): the MLP-shaped
scalar function of 64 inputs (two tanh layers of width 64, W ~ N(0, 1/64), b = 0
baked in as tape constants, output 0.5*||h||^2; ~25k tape slots), batch 65,536
points x ~ N(0, I), Rademacher v.  One step = a gradient sweep and a per-point HVP
sweep over the whole batch, FP32 (the throughput precision of that configuration).

* ``value``: points/s with inputs resident in HBM (device-pointer C ABI calls),
  CUDA events on the launching stream, L2 flushed between steps.
* ``e2e``: the same step through the host-buffer C ABI (ech_gradient_batch_f32 +
  ech_hvp_batch_points_f32): host->device copies of the inputs and device->host
  copies of the results are inside the timed region.
* ``roofline``: the dominant sweep kernel, algorithmic bytes per launch from the
  tape (``s*(2ni+no) + 2s*T_val`` per point for the gradient) over its event time.
* ``cpu_baseline``: the oracle (the reference's CPU sweeps restated in C++) on a
  bounded sample of the same workload, on all host cores.

``--impl reference`` times that CPU implementation alone as the reference arm.
Multi-GPU (torchrun): the global batch is world * 65,536 points and every rank
evaluates its own contiguous 65,536-point shard (points are independent, no
collective on the data path); timing is the max over ranks.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grad/HVP/Laplacian points/s (% roofline); time to 1% STDE error, learned vs plain"
UNIT = "points/s"
BATCH = 65536
N_IN = 64


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                mhz.append(float(s[0]))
                mx = float(s[1])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if s[4 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(mhz)}


def _workload(dtype, rank=0, world=1):
    """The tape and this rank's shard of the global batch (world * 65,536 points)."""
    from echidna_b200 import configs
    from echidna_b200.multi import rank_rows
    tape = configs.mlp(N_IN, 64, dtype=np.float64)
    seed = configs.SEEDS["mlp"]
    n = world * BATCH
    X = rank_rows(n, rank, world, seed, N_IN, lambda g, s: g.normal(size=s))
    V = rank_rows(n, rank, world, seed + 1, N_IN, lambda g, s: g.choice([-1.0, 1.0], size=s))
    return tape, X.astype(dtype), V.astype(dtype)


def cpu_reference(tape, X, V, budget_s: float, nthreads: int):
    """Oracle gradient + HVP (f64, the reference's CPU path) on a bounded sample."""
    from oracle.oracle import OracleTape
    o = OracleTape(tape)
    Xd = X.astype(np.float64)
    Vd = V.astype(np.float64)
    n = 64
    t0 = time.perf_counter()
    o.gradient(Xd[:n], nthreads)
    o.hvp(Xd[:n], Vd[:n], nthreads)
    dt = time.perf_counter() - t0
    n = int(min(len(Xd), max(n, n * budget_s / max(dt, 1e-6))))
    t0 = time.perf_counter()
    o.gradient(Xd[:n], nthreads)
    o.hvp(Xd[:n], Vd[:n], nthreads)
    dt = time.perf_counter() - t0
    return n / dt, n, dt


def run_reference(args):
    """Reference arm: the reference's CPU implementation (C++ restatement) alone."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as orc
    tape, X, V = _workload(np.float32)
    nth = os.cpu_count() or 1
    vals = []
    for _ in range(args.warmup):
        cpu_reference(tape, X, V, 0.5, nth)
    for _ in range(args.steps):
        v, n, dt = cpu_reference(tape, X, V, 3.0, nth)
        vals.append(v)
    value = float(np.median(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic", "scaling": "weak", "vs_baseline": None,
        "config": {"workload": "mlp n=64 width=64 (~25k-slot tape), gradient+HVP per point, batch 65536",
                   "batch": BATCH},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nth, "kind": "port",
                         "sample": f"{n} points of the batch per step, oracle gradient + per-point HVP (f64)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    from echidna_b200 import _lib
    from echidna_b200.gpu import CudaContext, GpuTapeData
    from echidna_b200.multi import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    lib = _lib.load()
    ctx = CudaContext.new(local)
    assert ctx is not None, "no CUDA device"

    tape, X, V = _workload(np.float32, rank, world)
    gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
    # a dedicated stream: the events below and the engine's launches must share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    assert sp != 0
    dX = torch.from_numpy(X).cuda()
    dV = torch.from_numpy(V).cuda()
    d_out = torch.empty(BATCH, device="cuda")
    d_g = torch.empty(BATCH * N_IN, device="cuda")
    d_g2 = torch.empty(BATCH * N_IN, device="cuda")
    d_h = torch.empty(BATCH * N_IN, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, device="cuda")

    def grad():
        st = lib.ech_gradient_batch_device(ctx._h, gt._h, 0, dX.data_ptr(), BATCH, d_out.data_ptr(), d_g.data_ptr(), sp)
        assert st == 0, _lib.last_error()

    def hvp():
        st = lib.ech_hvp_batch_device(ctx._h, gt._h, 0, dX.data_ptr(), 1, dV.data_ptr(), BATCH, d_g2.data_ptr(),
                                      d_h.data_ptr(), sp)
        assert st == 0, _lib.last_error()

    for _ in range(args.warmup):
        grad()
        hvp()
    torch.cuda.synchronize()
    assert lib.ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # device-resident timing, per kernel, L2 flushed between steps
    t_grad, t_hvp = [], []
    barrier()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            grad()
            e1.record(stream)
            hvp()
            e2.record(stream)
            e2.synchronize()
            t_grad.append(e0.elapsed_time(e1))
            t_hvp.append(e1.elapsed_time(e2))
        barrier()
    assert lib.ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()
    step_ms = float(np.sum(t_grad) + np.sum(t_hvp)) / args.steps
    if world > 1:
        step_ms = max_over_ranks(step_ms, "cuda")

    # end-to-end through the host-buffer ABI (pinned host buffers)
    hX = torch.from_numpy(X).pin_memory().numpy()
    hV = torch.from_numpy(V).pin_memory().numpy()
    ho = torch.empty(BATCH, pin_memory=True).numpy()
    hg = torch.empty(BATCH * N_IN, pin_memory=True).numpy()
    hg2 = torch.empty(BATCH * N_IN, pin_memory=True).numpy()
    hh = torch.empty(BATCH * N_IN, pin_memory=True).numpy()
    P = _lib.ptr

    def e2e_step():
        st = lib.ech_gradient_batch_f32(ctx._h, gt._h, P(hX), hX.size, BATCH, P(ho), ho.size, P(hg), hg.size)
        assert st == 0, _lib.last_error()
        st = lib.ech_hvp_batch_points_f32(ctx._h, gt._h, P(hX), hX.size, P(hV), hV.size, BATCH, P(hg2), hg2.size,
                                          P(hh), hh.size)
        assert st == 0, _lib.last_error()

    e2e_step()
    barrier()
    e2e_ms = []
    for _ in range(max(3, args.steps // 2)):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_step_ms = float(np.median(e2e_ms))
    if world > 1:
        e2e_step_ms = max_over_ranks(e2e_step_ms, "cuda")

    # roofline of the dominant kernel
    sg = ctx.plan_stats(gt, "gradient")
    sh = ctx.plan_stats(gt, "hvp")
    s = 4
    ni, no = N_IN, 1
    grad_bytes = BATCH * (s * (2 * ni + no) + 2 * s * sg["traj_values"])
    hvp_bytes = BATCH * (s * (4 * ni + no) + 2 * s * 2 * sh["traj_values"])
    g_ms = float(np.mean(t_grad))
    h_ms = float(np.mean(t_hvp))
    if g_ms >= h_ms:
        dom, dom_ms, dom_bytes, dom_flops = "gradient sweep", g_ms, grad_bytes, BATCH * (sg["flops_fwd"] + sg["flops_rev"])
    else:
        dom, dom_ms, dom_bytes, dom_flops = "hvp sweep", h_ms, hvp_bytes, BATCH * 4 * (sh["flops_fwd"] + sh["flops_rev"])
    peak, peak_kind = _peaks()
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(dom)

    value = world * BATCH / (step_ms * 1e-3)
    e2e_value = world * BATCH / (e2e_step_ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "mlp n=64 width=64 (~25k-slot tape): gradient + per-point HVP, Rademacher v",
                   "batch_per_gpu": BATCH, "l2": "flushed between steps (256 MiB write outside the events)",
                   "parallelism": f"points sharded, {world} rank(s)"},
        "gpu_launches": 2 * args.steps,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": dom_bytes, "launch_ms": dom_ms,
                     "fp32_ops_per_launch": dom_flops, "fp32_tflops": dom_flops / (dom_ms * 1e-3) / 1e12},
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int(hX.nbytes * 2 + hV.nbytes),
                "d2h_bytes_per_step": int(ho.nbytes + hg.nbytes + hg2.nbytes + hh.nbytes)},
        "clocks": clk.summary(),
        "detail": {"gradient_ms": g_ms, "hvp_ms": h_ms, "gradient_points_per_s": BATCH / (g_ms * 1e-3),
                   "hvp_points_per_s": BATCH / (h_ms * 1e-3), "plan_gradient": sg, "plan_hvp": sh,
                   "shape_gradient": ctx.launch_shape(gt, "gradient", BATCH),
                   "shape_hvp": ctx.launch_shape(gt, "hvp", BATCH)},
    }
    if rank == 0 and not args.no_cpu_baseline:
        nth = os.cpu_count() or 1
        v, n, dt = cpu_reference(tape, X, V, 10.0, nth)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": nth, "kind": "port",
                                "sample": f"{n} points: oracle gradient + per-point HVP (f64), {dt:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del gt
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
