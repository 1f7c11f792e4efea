"""Benchmark: batched BytecodeTape sweeps on B200 (one JSON line on rank 0).

Workloads (``--workload``, default ``mlp``):

* ``mlp`` — the configuration the headline metric is quoted on: the MLP-shaped
  scalar function of 64 inputs (two tanh layers of width 64, W ~ N(0, 1/64), b = 0
  baked in as tape constants, output 0.5*||h||^2; ~25k tape slots), 65,536 points
  x ~ N(0, I), Rademacher v.  One step = a gradient sweep and a per-point HVP sweep
  over the whole batch, FP32 (the throughput precision of that configuration).
* ``mlp64`` — the same MLP workload in FP64 (the configuration's parity precision).
* ``rosenbrock`` — extended Rosenbrock n=100 (bench-style recording), 1,024 points
  x ~ U[-2, 2]^100, f64; one step = one forward + gradient sweep.
* ``stde`` — f(x) = logsumexp(tanh(W x + b)), n=256, W in R^{512x256}; 16,384
  points, 64 Rademacher directions each from the device RNG, order-3 jets in FP32
  and a per-point Welford reduction in FP64; one step = one Laplacian batch.
* ``uneven`` — 64 different tapes with uneven lengths, input sizes and point
  counts; one step = gradient + per-point HVP of all of them in one persistent
  launch (FP32), compared in ``detail`` with one launch per tape and with a
  CUDA-graph replay of the persistent launch.
* ``learned`` — sparse STDE of a 1,024-input softplus chain with the learned
  proposal (BF16 tcgen05 MLP trained in setup on exact diagonals) vs uniform
  sampling; ``detail`` has the samples and wall time to 1 % relative error.

Reported per line:

* ``value``: points/s with inputs resident in HBM (device-pointer C ABI calls),
  CUDA events on the launching stream, L2 flushed between steps (256 MiB write
  outside the timed events).
* ``e2e``: the same step through the host-buffer C ABI with ordinary (pageable)
  numpy arrays, as a drop-in caller passes them: host->device copies of the
  inputs and device->host copies of the results are inside the timed region.
  ``detail.e2e_pinned_host_buffers`` repeats it with page-locked arrays.
* ``roofline``: the dominant kernel's algorithmic bytes per launch (the
  store-all model, from the tape) over its event time, against the measured HBM
  copy bandwidth (``frac``); beside it the algorithmic scalar ops per launch
  (``echidna_b200.opcost``, by value kind) against the CUDA-core pipe, and
  ``t_roof`` = max(bytes / HBM, ops / pipe) over the measured time.
* ``cpu_baseline``: the oracle (the reference's CPU sweeps restated in C++) on a
  bounded sample of the same workload, on all host cores.

``--impl reference`` times that CPU implementation alone as the reference arm.
Multi-GPU (torchrun): the global batch is world x (per-GPU batch) points and every
rank evaluates its own contiguous shard (points are independent, no collective
on the data path); timing is the max over ranks.
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
L2_FLUSH_BYTES = 256 * 1024 * 1024


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []       # (host time read, fields)
        self.proc = None
        self.window = None      # (start, end) host times of the timed region

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append((time.time(), parts))

    def mark(self, start: float, end: float):
        """The timed region; samples read up to 50 ms after its end belong to it."""
        self.window = (start, end + 0.05)

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
        for t, s in self.samples:
            if self.window and not (self.window[0] <= t <= self.window[1]):
                continue
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


# ───────────────────────────── workloads ─────────────────────────────────────

def _pinned(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


class MlpWorkload:
    name = "mlp"
    batch = 65536
    n = 64
    launches_per_step = 2
    f64 = False

    def __init__(self, rank, world):
        from echidna_b200 import configs
        from echidna_b200.multi import rank_rows
        self.tape = configs.mlp(self.n, 64, dtype=np.float64)
        self.dt = np.float64 if self.f64 else np.float32
        seed = configs.SEEDS["mlp"]
        total = world * self.batch
        self.X = rank_rows(total, rank, world, seed, self.n, lambda g, s: g.normal(size=s)).astype(self.dt)
        self.V = rank_rows(total, rank, world, seed + 1, self.n,
                           lambda g, s: g.choice([-1.0, 1.0], size=s)).astype(self.dt)

    def describe(self):
        return {"workload": "mlp n=64 width=64 (~25k-slot tape): gradient + per-point HVP, Rademacher v",
                "batch_per_gpu": self.batch}, "f64" if self.f64 else "f32"

    def setup(self, ctx, lib, torch, sp):
        from echidna_b200.gpu import GpuTapeData
        self.ctx, self.lib, self.sp = ctx, lib, sp
        self.gt = ctx.upload_tape_f64(self.tape) if self.f64 else ctx.upload_tape(
            GpuTapeData.from_tape_f64_lossy(self.tape))
        B, n = self.batch, self.n
        tdt = torch.float64 if self.f64 else torch.float32
        self.dX = torch.from_numpy(self.X).cuda()
        self.dV = torch.from_numpy(self.V).cuda()
        self.d_out = torch.empty(B, dtype=tdt, device="cuda")
        self.d_g = torch.empty(B * n, dtype=tdt, device="cuda")
        self.d_g2 = torch.empty(B * n, dtype=tdt, device="cuda")
        self.d_h = torch.empty(B * n, dtype=tdt, device="cuda")
        # end to end with ordinary (pageable) numpy arrays, as a drop-in caller passes
        # them; the pinned copies give the figure for callers that pin their buffers
        self.pX, self.pV = self.X.copy(), self.V.copy()
        self.po, self.pg = np.empty(B, self.dt), np.empty(B * n, self.dt)
        self.pg2, self.ph = np.empty(B * n, self.dt), np.empty(B * n, self.dt)
        self.hX, self.hV = _pinned(torch, self.X), _pinned(torch, self.V)
        self.ho = _pinned(torch, np.empty(B, self.dt))
        self.hg = _pinned(torch, np.empty(B * n, self.dt))
        self.hg2 = _pinned(torch, np.empty(B * n, self.dt))
        self.hh = _pinned(torch, np.empty(B * n, self.dt))

    def kernels(self):
        from echidna_b200 import _lib
        lib, ctx, gt, sp, f64 = self.lib, self.ctx, self.gt, self.sp, int(self.f64)

        def grad():
            st = lib.ech_gradient_batch_device(ctx._h, gt._h, f64, self.dX.data_ptr(), self.batch,
                                               self.d_out.data_ptr(), self.d_g.data_ptr(), sp)
            assert st == 0, _lib.last_error()

        def hvp():
            st = lib.ech_hvp_batch_device(ctx._h, gt._h, f64, self.dX.data_ptr(), 1, self.dV.data_ptr(), self.batch,
                                          self.d_g2.data_ptr(), self.d_h.data_ptr(), sp)
            assert st == 0, _lib.last_error()
        return [("gradient sweep", grad), ("hvp sweep", hvp)]

    def _e2e(self, X, V, o, g, g2, h):
        from echidna_b200 import _lib
        lib, ctx, gt, P, B = self.lib, self.ctx, self.gt, _lib.ptr, self.batch
        sfx = "f64" if self.f64 else "f32"
        st = getattr(lib, f"ech_gradient_batch_{sfx}")(ctx._h, gt._h, P(X), X.size, B, P(o), o.size, P(g), g.size)
        assert st == 0, _lib.last_error()
        st = getattr(lib, f"ech_hvp_batch_points_{sfx}")(ctx._h, gt._h, P(X), X.size, P(V), V.size, B, P(g2),
                                                           g2.size, P(h), h.size)
        assert st == 0, _lib.last_error()

    def e2e_step(self):
        self._e2e(self.pX, self.pV, self.po, self.pg, self.pg2, self.ph)

    def e2e_step_pinned(self):
        self._e2e(self.hX, self.hV, self.ho, self.hg, self.hg2, self.hh)

    def io_bytes(self):
        return (int(self.hX.nbytes * 2 + self.hV.nbytes),
                int(self.ho.nbytes + self.hg.nbytes + self.hg2.nbytes + self.hh.nbytes))

    def roofline_inputs(self, kernel):
        from echidna_b200 import opcost
        s, ni, no, B = (8 if self.f64 else 4), self.n, 1, self.batch
        if kernel == "gradient sweep":
            st = self.ctx.plan_stats(self.gt, "gradient")
            return B * (s * (2 * ni + no) + 2 * s * st["traj_values"]), B * opcost.sweep_cost(self.tape, "gradient")[0]
        st = self.ctx.plan_stats(self.gt, "hvp")
        return B * (s * (4 * ni + no) + 2 * s * 2 * st["traj_values"]), B * opcost.sweep_cost(self.tape, "hvp")[0]

    def detail(self):
        return {"plan_gradient": self.ctx.plan_stats(self.gt, "gradient"),
                "plan_hvp": self.ctx.plan_stats(self.gt, "hvp"),
                "shape_gradient": self.ctx.launch_shape(self.gt, "gradient", self.batch),
                "shape_hvp": self.ctx.launch_shape(self.gt, "hvp", self.batch)}

    def accuracy(self, k=256):
        """The timed launches' gradients and HVPs of the first k points against the
        FP64 oracle (error = max |GPU - FP64| / max |FP64| per quantity), beside the
        same-precision oracle's own error.  Run in the CPU-baseline leg, after timing."""
        from oracle.oracle import OracleTape
        n = self.n
        g = self.d_g.view(self.batch, n)[:k].double().cpu().numpy()
        g2 = self.d_g2.view(self.batch, n)[:k].double().cpu().numpy()
        h = self.d_h.view(self.batch, n)[:k].double().cpu().numpy()
        X, V = self.X[:k].astype(np.float64), self.V[:k].astype(np.float64)
        o64 = OracleTape(self.tape, dtype=np.float64)
        _, rg = o64.gradient(X)
        rg2, rh = o64.hvp(X, V)

        def err(a, ref):
            return float(np.max(np.abs(a - ref)) / max(np.max(np.abs(ref)), 1e-300))
        out = {"reference": "oracle (FP64 CPU tape) on the first %d points" % k,
               "gradient_vs_fp64": err(g, rg), "hvp_gradient_vs_fp64": err(g2, rg2), "hvp_vs_fp64": err(h, rh)}
        if not self.f64:
            o32 = OracleTape(self.tape, dtype=np.float32)
            _, sg = o32.gradient(X.astype(np.float32))
            _, sh = o32.hvp(X.astype(np.float32), V.astype(np.float32))
            out["fp32_oracle_gradient_vs_fp64"] = err(sg.astype(np.float64), rg)
            out["fp32_oracle_hvp_vs_fp64"] = err(sh.astype(np.float64), rh)
        return out

    def cpu_reference(self, budget_s, nthreads, dtype=np.float64):
        from oracle.oracle import OracleTape
        o = OracleTape(self.tape, dtype=dtype)
        Xd, Vd = self.X.astype(dtype), self.V.astype(dtype)
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
        prec = "f64" if dtype == np.float64 else "f32"
        return n / dt, f"{n} points of the batch: oracle gradient + per-point HVP ({prec}), {dt:.1f} s"


class Mlp64Workload(MlpWorkload):
    """The same MLP workload in FP64 (the configuration's parity precision)."""
    name = "mlp64"
    f64 = True


class RosenbrockWorkload:
    name = "rosenbrock"
    batch = 1024
    n = 100
    launches_per_step = 1

    def __init__(self, rank, world):
        from echidna_b200 import configs
        from echidna_b200.multi import rank_rows
        self.tape = configs.rosenbrock(self.n)
        self.X = rank_rows(world * self.batch, rank, world, configs.SEEDS["rosenbrock"], self.n,
                           lambda g, s: g.uniform(-2.0, 2.0, size=s))

    def describe(self):
        return {"workload": "extended Rosenbrock n=100 (1,091-slot tape): forward value + gradient",
                "batch_per_gpu": self.batch}, "f64"

    def setup(self, ctx, lib, torch, sp):
        self.ctx, self.lib, self.sp = ctx, lib, sp
        self.gt = ctx.upload_tape_f64(self.tape)
        B, n = self.batch, self.n
        self.dX = torch.from_numpy(self.X).cuda()
        self.d_out = torch.empty(B, dtype=torch.float64, device="cuda")
        self.d_g = torch.empty(B * n, dtype=torch.float64, device="cuda")
        self.pX, self.po, self.pg = self.X.copy(), np.empty(B), np.empty(B * n)
        self.hX = _pinned(torch, self.X)
        self.ho = _pinned(torch, np.empty(B))
        self.hg = _pinned(torch, np.empty(B * n))

    def kernels(self):
        from echidna_b200 import _lib

        def grad():
            st = self.lib.ech_gradient_batch_device(self.ctx._h, self.gt._h, 1, self.dX.data_ptr(), self.batch,
                                                    self.d_out.data_ptr(), self.d_g.data_ptr(), self.sp)
            assert st == 0, _lib.last_error()
        return [("gradient sweep", grad)]

    def _e2e(self, X, o, g):
        from echidna_b200 import _lib
        P = _lib.ptr
        st = self.lib.ech_gradient_batch_f64(self.ctx._h, self.gt._h, P(X), X.size, self.batch, P(o), o.size, P(g),
                                             g.size)
        assert st == 0, _lib.last_error()

    def e2e_step(self):
        self._e2e(self.pX, self.po, self.pg)

    def e2e_step_pinned(self):
        self._e2e(self.hX, self.ho, self.hg)

    def io_bytes(self):
        return int(self.hX.nbytes), int(self.ho.nbytes + self.hg.nbytes)

    def roofline_inputs(self, kernel):
        from echidna_b200 import opcost
        st = self.ctx.plan_stats(self.gt, "gradient")
        s, B = 8, self.batch
        return B * (s * (2 * self.n + 1) + 2 * s * st["traj_values"]), B * opcost.sweep_cost(self.tape, "gradient")[0]

    def detail(self):
        return {"plan_gradient": self.ctx.plan_stats(self.gt, "gradient"),
                "shape_gradient": self.ctx.launch_shape(self.gt, "gradient", self.batch)}

    def cpu_reference(self, budget_s, nthreads):
        from oracle.oracle import OracleTape
        o = OracleTape(self.tape)
        reps, t0 = 0, time.perf_counter()
        while True:
            o.gradient(self.X, nthreads)
            reps += 1
            dt = time.perf_counter() - t0
            if dt >= budget_s or reps >= 100000:
                break
        return reps * self.batch / dt, f"{reps} x {self.batch} points: oracle forward + gradient (f64), {dt:.1f} s"


class StdeWorkload:
    name = "stde"
    batch = 16384
    n = 256
    S = 64
    launches_per_step = 2

    def __init__(self, rank, world):
        from echidna_b200 import configs
        from echidna_b200.multi import rank_rows
        self.tape = configs.logsumexp_tanh(self.n, 512)
        self.seed = configs.SEEDS["logsumexp_tanh"]
        self.X = rank_rows(world * self.batch, rank, world, self.seed, self.n,
                           lambda g, s: g.normal(size=s)).astype(np.float32)

    def describe(self):
        return {"workload": "STDE Laplacian: logsumexp(tanh(Wx+b)), n=256, W 512x256 (~395k-slot tape), "
                            "S=64 device-RNG Rademacher directions, order-3 jets (FP32), FP64 Welford",
                "batch_per_gpu": self.batch, "directions": self.S}, "f32"

    def setup(self, ctx, lib, torch, sp):
        from echidna_b200 import _lib
        from echidna_b200.gpu import GpuTapeData
        self.ctx, self.lib, self.sp = ctx, lib, sp
        self.gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(self.tape))
        self.dX = torch.from_numpy(self.X).cuda()
        self.d_res = torch.empty(self.batch * 5, dtype=torch.float64, device="cuda")
        self.pX = self.X.copy()
        self.hX = _pinned(torch, self.X)
        self.h_res = (_lib.EstimatorResultC * self.batch)()

    def kernels(self):
        from echidna_b200 import _lib

        def lap():
            st = self.lib.ech_laplacian_batch_device(self.ctx._h, self.gt._h, 0, self.dX.data_ptr(), self.batch, None,
                                                     self.S, 2, self.seed, self.d_res.data_ptr(), self.sp)
            assert st == 0, _lib.last_error()
        return [("taylor-3 sweep + reduction", lap)]

    def _e2e(self, X):
        from echidna_b200 import _lib
        st = self.lib.ech_laplacian_batch_f32(self.ctx._h, self.gt._h, _lib.ptr(X), X.size, self.batch,
                                              None, 0, self.S, 2, self.seed, self.h_res)
        assert st == 0, _lib.last_error()

    def e2e_step(self):
        self._e2e(self.pX)

    def e2e_step_pinned(self):
        self._e2e(self.hX)

    def io_bytes(self):
        return int(self.hX.nbytes), int(self.batch * 40)

    def roofline_inputs(self, kernel):
        from echidna_b200 import opcost
        s, K = 4, 3
        units = self.batch * self.S
        # per unit: x amortised over the S directions, no direction bytes (device RNG), K coefficients out
        return int(units * s * (self.n / self.S + K)), units * opcost.sweep_cost(self.tape, "taylor", K)[0]

    def detail(self):
        return {"plan_taylor3": self.ctx.plan_stats(self.gt, "taylor", 3),
                "plan_taylor3_input_direct": self.ctx.plan_stats(self.gt, "taylor_direct", 3),
                "shape_taylor3": self.ctx.launch_shape(self.gt, "taylor", self.batch * self.S, 3)}

    accuracy_points = 256

    def extra(self, torch, stream, flush, steps):
        """Accuracy on a 256-point subset of the batch: the FP32 estimates against the
        exact Hessian trace of the oracle's dense tape Hessian (FP64), as relative
        error and z-score; and each FP32 option against the FP64 sweep with the same
        device directions (an FP64 GPU run, parity-tested against the oracle)."""
        import concurrent.futures as cf
        from echidna_b200 import stde_gpu
        from oracle.oracle import OracleTape
        k = self.accuracy_points
        X = self.X[:k]
        o = OracleTape(self.tape)
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(os.cpu_count() or 1) as ex:
            traces = np.array(list(ex.map(lambda x: float(np.trace(o.hessian(x.astype(np.float64))[2])), X)))
        t_oracle = time.perf_counter() - t0
        g64 = self.ctx.upload_tape_f64(self.tape)
        ref = stde_gpu.laplacian_batch(self.ctx, g64, X.astype(np.float64), self.S, None,
                                       stde_gpu.DIR_RADEMACHER, seed=self.seed)["estimate"]
        modes = {"fp32 jets, fp64 welford (default)": 0,
                 "fp32 jets, fp32 welford": self.ctx.FP32_PLAIN_MEANS,
                 "fp32 jets, compensated fp32 means": self.ctx.FP32_COMPENSATED_MEANS,
                 "compensated fp32 jets and means": self.ctx.FP32_COMPENSATED_JETS | self.ctx.FP32_COMPENSATED_MEANS}
        out = {}
        for name, flags in modes.items():
            self.ctx.set_fp32_mode(flags)
            r = stde_gpu.laplacian_batch(self.ctx, self.gt, X, self.S, None, stde_gpu.DIR_RADEMACHER, seed=self.seed)
            rel64 = np.abs(r["estimate"] - ref) / np.abs(ref)
            entry = {"vs_fp64_sweep_rel_err_median": float(np.median(rel64)), "vs_fp64_sweep_rel_err_max":
                     float(np.max(rel64))}
            if flags == 0:
                z = (r["estimate"] - traces) / r["standard_error"]
                rel = np.abs(r["estimate"] - traces) / np.abs(traces)
                entry.update({"vs_exact_trace_rel_err_median": float(np.median(rel)),
                              "vs_exact_trace_rel_err_max": float(np.max(rel)),
                              "z_abs_max": float(np.max(np.abs(z))), "z_mean": float(np.mean(z)),
                              "z_std": float(np.std(z))})
            out[name] = entry
        self.ctx.set_fp32_mode(0)
        rel64 = np.abs(ref - traces) / np.abs(traces)
        return {"accuracy_256_points": {"exact_trace": "trace of the oracle's dense tape Hessian (FP64), "
                                                       f"{t_oracle:.1f} s on the host",
                                        "fp64_sweep_vs_exact_trace_rel_err_median": float(np.median(rel64)),
                                        **out}}

    def cpu_reference(self, budget_s, nthreads):
        from oracle.oracle import OracleTape
        o = OracleTape(self.tape)
        rng = np.random.default_rng(self.seed)
        dirs = rng.choice([-1.0, 1.0], size=(self.S, self.n))
        Xd = self.X.astype(np.float64)
        n = 4
        t0 = time.perf_counter()
        o.laplacian_stats_batch(Xd[:n], dirs, nthreads)
        dt = time.perf_counter() - t0
        n = int(min(len(Xd), max(n, n * budget_s / max(dt, 1e-6))))
        t0 = time.perf_counter()
        o.laplacian_stats_batch(Xd[:n], dirs, nthreads)
        dt = time.perf_counter() - t0
        return n / dt, f"{n} points x 64 directions: oracle stde::laplacian per point (f64), {dt:.1f} s"


class UnevenWorkload:
    """64 different tapes (Rosenbrock, Ackley-type, random DAGs of 200-20,000 ops), input
    sizes 2-512 and 1-100,000 points each: gradient + per-point HVP of all of them in one
    persistent launch (FP32).  ``detail`` adds one launch per tape and a CUDA-graph replay."""
    name = "uneven"
    launches_per_step = 1

    def __init__(self, rank, world):
        from echidna_b200 import configs
        self.seed = configs.SEEDS["uneven"]
        self.suite = configs.uneven_suite(64, self.seed)
        rng = np.random.default_rng([self.seed, rank])
        self.data = []
        for _, tape, n in self.suite:
            ni = tape.num_inputs
            self.data.append((rng.uniform(-1.0, 1.0, size=(n, ni)).astype(np.float32),
                              rng.choice([-1.0, 1.0], size=(n, ni)).astype(np.float32)))
        self.batch = sum(n for _, _, n in self.suite)

    def describe(self):
        return {"workload": "uneven batch: 64 tapes (Rosenbrock / Ackley-type / random DAGs 200-20k ops), "
                            "dims 2-512, 1-100k points each; gradient + per-point HVP in one persistent launch",
                "points_per_gpu": self.batch, "tapes": len(self.suite)}, "f32"

    def setup(self, ctx, lib, torch, sp):
        from echidna_b200.gpu import GpuTapeData, MultiTapeHvp
        self.ctx, self.lib, self.sp, self.torch = ctx, lib, sp, torch
        self.jobs = []
        for (_, tape, n), (x, v) in zip(self.suite, self.data):
            gt = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(tape))
            dx, dv = torch.from_numpy(x).cuda(), torch.from_numpy(v).cuda()
            g, h = torch.empty_like(dx), torch.empty_like(dx)
            hx, hv = _pinned(torch, x), _pinned(torch, v)
            hg, hh = _pinned(torch, np.empty_like(x)), _pinned(torch, np.empty_like(x))
            self.jobs.append((tape, gt, n, dx, dv, g, h, hx, hv, hg, hh))
        torch.cuda.synchronize()
        items = [(gt, dx.data_ptr(), dv.data_ptr(), n, g.data_ptr(), h.data_ptr())
                 for _, gt, n, dx, dv, g, h, *_ in self.jobs]
        self.multi = MultiTapeHvp(ctx, items, f64=False, autotune=True)
        # end to end: the tapes in four groups of about equal bytes, each its own
        # many-tape launch on its own stream, so one group's copies overlap the
        # others' sweeps
        order = sorted(range(len(self.jobs)), key=lambda k: -self.jobs[k][7].nbytes)
        groups, load = [[] for _ in range(4)], [0] * 4
        for k in order:
            gi = int(np.argmin(load))
            groups[gi].append(k)
            load[gi] += self.jobs[k][7].nbytes
        self.e2e_groups = [(ks, MultiTapeHvp(ctx, [items[k] for k in ks], f64=False, autotune=True),
                            torch.cuda.Stream()) for ks in groups if ks]

    def kernels(self):
        return [("multi-tape launch", lambda: self.multi.launch(self.sp))]

    def per_tape(self):
        from echidna_b200 import _lib
        for _, gt, n, dx, dv, g, h, *_ in self.jobs:
            st = self.lib.ech_hvp_batch_device(self.ctx._h, gt._h, 0, dx.data_ptr(), 1, dv.data_ptr(), n,
                                               g.data_ptr(), h.data_ptr(), self.sp)
            assert st == 0, _lib.last_error()

    def extra(self, torch, stream, flush, steps):
        """One launch per tape, and the multi launch replayed from a CUDA graph."""
        for _ in range(3):
            self.per_tape()
        torch.cuda.synchronize()
        t_per = []
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            self.per_tape()
            e1.record(stream)
            e1.synchronize()
            t_per.append(e0.elapsed_time(e1))
        graph = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream()
        with torch.cuda.graph(graph, stream=cap, capture_error_mode="thread_local"):
            self.multi.launch(cap.cuda_stream)
        graph.replay()
        torch.cuda.synchronize()
        t_graph = []
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            graph.replay()
            e1.record(stream)
            e1.synchronize()
            t_graph.append(e0.elapsed_time(e1))
        del graph
        return {"one launch per tape ms": float(np.mean(t_per)), "graph replay ms": float(np.mean(t_graph)),
                "multi_shape": self.multi.info()}

    def e2e_step(self):
        """Through the many-tape API, pipelined: per group of tapes, on the group's
        stream, its points and directions copied in from pinned host memory, one
        persistent launch, its gradients and HVPs copied back; then a synchronise."""
        torch = self.torch
        for ks, multi, st in self.e2e_groups:
            with torch.cuda.stream(st):
                for k in ks:
                    _, _, _, dx, dv, _, _, hx, hv, _, _ = self.jobs[k]
                    dx.copy_(torch.from_numpy(hx), non_blocking=True)
                    dv.copy_(torch.from_numpy(hv), non_blocking=True)
                multi.launch(st.cuda_stream)
                for k in ks:
                    _, _, _, _, _, g, h, _, _, hg, hh = self.jobs[k]
                    torch.from_numpy(hg).copy_(g, non_blocking=True)
                    torch.from_numpy(hh).copy_(h, non_blocking=True)
        for _, _, st in self.e2e_groups:
            st.synchronize()

    def io_bytes(self):
        h2d = sum(j[7].nbytes + j[8].nbytes for j in self.jobs)
        d2h = sum(j[9].nbytes + j[10].nbytes for j in self.jobs)
        return int(h2d), int(d2h)

    def roofline_inputs(self, kernel):
        from echidna_b200 import opcost
        s, total_b, total_f = 4, 0, 0
        for tape, gt, n, *_ in self.jobs:
            st = self.ctx.plan_stats(gt, "hvp")
            ni = tape.num_inputs
            total_b += n * (s * (4 * ni + 1) + 2 * s * 2 * st["traj_values"])
            total_f += n * opcost.sweep_cost(tape, "hvp")[0]
        return total_b, total_f

    def detail(self):
        return {}

    def cpu_reference(self, budget_s, nthreads):
        from oracle.oracle import OracleTape
        orcs = [OracleTape(tape) for _, tape, _ in self.suite]

        def run(k):
            pts = 0
            t0 = time.perf_counter()
            for o, (x, v), (_, _, n) in zip(orcs, self.data, self.suite):
                m = min(n, k)
                o.hvp(x[:m].astype(np.float64), v[:m].astype(np.float64), nthreads)
                pts += m
            return pts, time.perf_counter() - t0
        pts, dt = run(4)
        k = int(max(4, 4 * budget_s / max(dt, 1e-6)))
        pts, dt = run(k)
        return pts / dt, f"{pts} points (up to {k} per tape): oracle gradient + per-point HVP (f64), {dt:.1f} s"


class LearnedWorkload:
    """C5: sparse STDE trace of f = sum a_i softplus(x_i x_{i+1}) + sum a_i cos x_i (n = 1,024,
    a_i log-uniform in [1e-3, 1e3]) with the learned proposal vs uniform sampling.  Setup
    draws the configured 1,048,576 training points on the device, labels them with exact FP64
    diagonals (one per-point HVP per color of the Hessian's tridiagonal pattern: two HVPs per
    point) and trains the 1024-256-256-1024 BF16 MLP on the GPU; the held-out points' diagonals
    come from order-3 jets along every e_j and are compared with the colored HVPs.  The timed
    step is the learned estimator (MLP + 256 sampled jets per point, FP32 jets, FP64 Welford)
    over 1,024 held-out points.  ``detail`` gives the samples and wall time each proposal
    needs for 1 % relative error."""
    name = "learned"
    n = 1024
    batch = 1024          # held-out points per timed step
    S = 256               # samples per point in the timed step
    launches_per_step = 10  # MLP: 3 conversions, 3 GEMMs, softmax; sampler, jet sweep, reduction
    n_train = 1 << 20
    n_eval = 1024
    train_steps = 4000
    train_batch = 1024

    def __init__(self, rank, world):
        from echidna_b200 import configs
        self.seed = configs.SEEDS["softplus_chain"]
        self.rank = rank
        self.tape = configs.softplus_chain(self.n)
        rng = np.random.default_rng([self.seed, rank])
        self.Xev = rng.normal(size=(self.n_eval, self.n))

    def describe(self):
        return {"workload": "learned STDE proposal: softplus-chain n=1024, MLP 1024-256-256-1024 (BF16 tcgen05, "
                            "FP32 accumulation) trained on exact FP64 diagonals; learned vs uniform sparse STDE",
                "eval_points": self.batch, "samples_per_point_in_step": self.S,
                "training_points": self.n_train, "training_steps": self.train_steps,
                "training_batch": self.train_batch}, "f32"

    def setup(self, ctx, lib, torch, sp):
        from echidna_b200 import learned
        from echidna_b200.gpu import GpuTapeData
        from echidna_b200.sparse import detect_sparsity
        self.ctx, self.lib, self.sp, self.torch = ctx, lib, sp, torch
        self.g64 = ctx.upload_tape_f64(self.tape)
        self.g32 = ctx.upload_tape(GpuTapeData.from_tape_f64_lossy(self.tape))
        coloring = learned.diagonal_coloring(detect_sparsity(self.tape))
        self.num_colors = coloring[1]
        # labels and training run on the default stream, before the timed stream is used
        with torch.cuda.stream(torch.cuda.default_stream()):
            g = torch.Generator(device="cuda").manual_seed(self.seed + self.rank)
            xtr = torch.randn((self.n_train, self.n), dtype=torch.float64, device="cuda", generator=g)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            d = learned.colored_diagonals(ctx, self.g64, xtr, coloring)
            torch.cuda.synchronize()
            self.t_labels = time.perf_counter() - t0
            q = learned.target_distribution(d)
            del d
            xf = xtr.float()
            del xtr
            t0 = time.perf_counter()
            self.mlp = learned.ProposalMLP(ctx, self.n, 256, self.n, seed=self.seed)
            self.losses = []
            for _ in range(self.train_steps):
                rows = torch.randint(0, self.n_train, (self.train_batch,), device="cuda", generator=g)
                self.losses.append(self.mlp.train_step(xf[rows].contiguous(), q[rows].contiguous(), lr=1e-3))
            torch.cuda.synchronize()
            self.t_train = time.perf_counter() - t0
            del xf, q
            xev = torch.tensor(self.Xev, device="cuda")
            t0 = time.perf_counter()
            d_ev = learned.exact_diagonals(ctx, self.g64, xev)
            torch.cuda.synchronize()
            self.t_eval_jets = time.perf_counter() - t0
            d_col = learned.colored_diagonals(ctx, self.g64, xev, coloring)
            scale = d_ev.abs().amax(dim=1, keepdim=True)
            self.label_diff = float(((d_col - d_ev).abs() / scale).max())
            self.d_eval = d_ev.cpu().numpy()
            self.xev32 = xev.float().contiguous()
            self.p_eval = self.mlp.probs(self.xev32).cpu().numpy()
            torch.cuda.synchronize()
        self.probs = torch.empty((self.batch, self.n), dtype=torch.float32, device="cuda")
        self.res = torch.empty((self.batch, 5), dtype=torch.float64, device="cuda")
        self.hX = _pinned(torch, self.Xev.astype(np.float32))
        self.h_res = _pinned(torch, np.empty((self.batch, 5)))

    def _learned(self, S):
        from echidna_b200 import learned
        self.mlp.probs(self.xev32, out=self.probs, stream=self.sp)
        learned.sparse_trace(self.ctx, self.g32, self.xev32, self.probs, S, self.seed, self.res, stream=self.sp)

    def _uniform(self, S):
        from echidna_b200 import learned
        learned.sparse_trace(self.ctx, self.g32, self.xev32, None, S, self.seed, self.res, stream=self.sp)

    def kernels(self):
        return [("learned estimator (MLP + sampled jets)", lambda: self._learned(self.S))]

    def extra(self, torch, stream, flush, steps):
        from echidna_b200 import learned
        ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))  # noqa: E731
        def timed(fn):
            fn()
            torch.cuda.synchronize()
            ts = []
            for _ in range(steps):
                flush.zero_()
                e0, e1 = ev()
                e0.record(stream)
                fn()
                e1.record(stream)
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            return float(np.mean(ts))
        gemm = self._gemm_rates(torch, stream, timed)
        t_learn = timed(lambda: self._learned(self.S))
        t_unif = timed(lambda: self._uniform(self.S))
        t_mlp = timed(lambda: self.mlp.probs(self.xev32, out=self.probs, stream=self.sp))
        s_u, _, T = learned.samples_to_tolerance(self.d_eval, None)
        s_l, _, _ = learned.samples_to_tolerance(self.d_eval, self.p_eval)
        s_b, _, _ = learned.samples_to_tolerance(self.d_eval, np.abs(self.d_eval))
        per_sample_l = (t_learn - t_mlp) / (self.batch * self.S)   # ms per sampled jet
        per_sample_u = t_unif / (self.batch * self.S)
        med_l, med_u = float(np.median(s_l)), float(np.median(s_u))
        time_l = med_l * per_sample_l + t_mlp / self.batch
        time_u = med_u * per_sample_u
        # empirical check on 32 points at their own 1% sample counts (capped)
        k = 32
        S_chk = int(min(np.ceil(med_l), 200000))
        x = self.xev32[:k].contiguous()
        pr = self.mlp.probs(x)
        r = learned.as_records(learned.sparse_trace(self.ctx, self.g32, x, pr, S_chk, self.seed + 1))
        rel = np.abs(r["estimate"] - T[:k]) / np.abs(T[:k])
        return {"samples_to_1pct_median": {"uniform": med_u, "learned": med_l, "best_possible": float(np.median(s_b))},
                "time_to_1pct_ms_per_point_median": {"uniform": time_u, "learned": time_l,
                                                     "learned_speedup": time_u / time_l},
                "per_sample_jet_us": {"uniform": per_sample_u * 1e3, "learned": per_sample_l * 1e3},
                "mlp_forward_ms_per_1024_points": t_mlp, "uniform_step_ms": t_unif,
                "check_32_points_at_median_samples": {"samples": S_chk,
                                                      "median_relative_error": float(np.median(rel))},
                "labels": {"points": self.n_train, "hvps_per_point": self.num_colors, "seconds": self.t_labels,
                           "eval_1024_points_by_jets_s": self.t_eval_jets,
                           "max_rel_diff_colored_hvp_vs_jets": self.label_diff},
                "training_s": self.t_train, "loss_first_last": [self.losses[0], self.losses[-1]],
                "gemm_bf16_tcgen05": gemm}

    def _gemm_rates(self, torch, stream, timed):
        """TFLOP/s of the proposal's tensor-core GEMM (``ech_gemm_bf16``) at the MLP's
        first-layer shape (batch 1,024) and at 8192^3, against the measured cuBLAS peak."""
        import ctypes
        from echidna_b200 import _lib as _lib_mod
        lib = _lib_mod.load()
        pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
        peak, src = 1590.0, "fallback"
        if os.path.exists(pk):
            with open(pk) as f:
                peak, src = float(json.load(f).get("bf16_tflops", 1590.0)), "measured (cuBLAS bf16, burst)"
        out = {"peak_bf16_tflops": peak, "peak_source": src}
        for (M, N, K) in [(1024, 256, 1024), (8192, 8192, 8192)]:
            g = torch.Generator(device="cuda").manual_seed(M + N + K)
            A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
            B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
            C = torch.empty(M, N, device="cuda", dtype=torch.float32)
            st = ctypes.c_void_p(stream.cuda_stream)

            def run():
                r = lib.ech_gemm_bf16(self.ctx._h, A.data_ptr(), B.data_ptr(), C.data_ptr(), None, M, N, K, K, K,
                                      N, st)
                if r != 0:
                    raise RuntimeError(_lib_mod.last_error())
            ms = timed(run)
            ref = (A[:64].float() @ B.float().T)
            err = float((C[:64] - ref).abs().max() / ref.abs().max().clamp_min(1.0))
            tf = 2.0 * M * N * K / (ms * 1e-3) / 1e12
            out[f"{M}x{N}x{K}"] = {"ms": ms, "tflops": tf,
                                   "frac_of_peak": tf / peak,
                                   "max_rel_err_vs_fp32_first_64_rows": err}
            del A, B, C
        return out

    def e2e_step(self):
        torch = self.torch
        x = torch.from_numpy(self.hX).to("cuda", non_blocking=True)
        from echidna_b200 import learned
        pr = self.mlp.probs(x, out=self.probs, stream=self.sp)
        learned.sparse_trace(self.ctx, self.g32, x, pr, self.S, self.seed, self.res, stream=self.sp)
        self.h_res_t = self.res.to("cpu", non_blocking=True)
        torch.cuda.current_stream().synchronize()

    def io_bytes(self):
        return int(self.hX.nbytes), int(self.batch * 40)

    def roofline_inputs(self, kernel):
        from echidna_b200 import opcost
        units = self.batch * self.S
        return int(units * 4 * (self.n / self.S + 3)), units * opcost.sweep_cost(self.tape, "taylor", 3)[0]

    def detail(self):
        return {"plan_taylor3": self.ctx.plan_stats(self.g32, "taylor", 3)}

    def cpu_reference(self, budget_s, nthreads):
        """Uniform sparse STDE on the reference CPU path (diagonal_kth_order_stochastic, k=2)."""
        from oracle.oracle import OracleTape
        o = OracleTape(self.tape)
        rng = np.random.default_rng(self.seed)
        pts, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget_s / 4 and pts < 256:
            o.diagonal_kth_order_stochastic(self.Xev[pts], 2, rng.integers(0, self.n, size=self.S))
            pts += 1
        dt = time.perf_counter() - t0
        return pts / dt, f"{pts} points x {self.S} uniform samples: oracle diagonal_kth_order_stochastic (k=2, f64, 1 thread), {dt:.1f} s"


WORKLOADS = {"mlp": MlpWorkload, "mlp64": Mlp64Workload, "rosenbrock": RosenbrockWorkload, "stde": StdeWorkload, "uneven": UnevenWorkload,
             "learned": LearnedWorkload}


# ───────────────────────────── arms ──────────────────────────────────────────

def run_reference(args):
    """Reference arm: the reference's CPU implementation (C++ restatement) alone."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = WORKLOADS[args.workload](0, 1)
    nth = os.cpu_count() or 1
    for _ in range(args.warmup):
        wl.cpu_reference(0.3, nth)
    vals, sample = [], ""
    for _ in range(args.steps):
        v, sample = wl.cpu_reference(3.0, nth)
        vals.append(v)
    value = float(np.median(vals))
    cfg, dtype = wl.describe()
    detail = {}
    if dtype == "f32" and "dtype" in wl.cpu_reference.__code__.co_varnames:
        v32, s32 = wl.cpu_reference(3.0, nth, dtype=np.float32)
        detail["same_precision_f32"] = {"value": v32, "unit": UNIT, "sample": s32}
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic", "scaling": "weak", "vs_baseline": None, "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nth, "kind": "port", "sample": sample,
                         "cpu_model": _cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if detail:
        line["detail"] = detail
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="mlp", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-one-step", action="store_true",
                    help="after the warm-up, run one step between cudaProfilerStart/Stop and exit "
                         "(for ncu --profile-from-start off); prints no JSON line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    from echidna_b200 import _lib
    from echidna_b200.gpu import CudaContext
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

    wl = WORKLOADS[args.workload](rank, world)
    # a dedicated stream: the events below and the engine's launches must share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sp = stream.cuda_stream
    assert sp != 0
    wl.setup(ctx, lib, torch, sp)
    kernels = wl.kernels()
    flush = torch.empty(L2_FLUSH_BYTES // 4, device="cuda")

    clk = ClockSampler(local).__enter__()  # sampling from the warm-up on; only the timed region is kept
    for _ in range(args.warmup):
        for _, k in kernels:
            k()
    torch.cuda.synchronize()
    assert lib.ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()
    if args.profile_one_step:
        clk.__exit__(None, None, None)
        torch.cuda.cudart().cudaProfilerStart()
        for _, k in kernels:
            k()
        torch.cuda.synchronize()
        assert lib.ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()
        torch.cuda.cudart().cudaProfilerStop()
        print(f"profiled one step of {args.workload}: " + ", ".join(name for name, _ in kernels), flush=True)
        del kernels, wl
        ctx.close()
        return 0

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # device-resident timing, per kernel, L2 flushed between steps
    times = {name: [] for name, _ in kernels}
    barrier()
    t_start = time.time()
    for _ in range(args.steps):
        flush.zero_()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(kernels) + 1)]
        ev[0].record(stream)
        for i, (_, k) in enumerate(kernels):
            k()
            ev[i + 1].record(stream)
        ev[-1].synchronize()
        for i, (name, _) in enumerate(kernels):
            times[name].append(ev[i].elapsed_time(ev[i + 1]))
    barrier()
    clk.mark(t_start, time.time())
    time.sleep(0.1)
    clk.__exit__(None, None, None)
    assert lib.ech_ctx_synchronize(ctx._h) == 0, _lib.last_error()
    step_ms = float(sum(np.sum(v) for v in times.values())) / args.steps
    if world > 1:
        step_ms = max_over_ranks(step_ms, "cuda")

    extra = wl.extra(torch, stream, flush, args.steps) if hasattr(wl, "extra") else {}

    # end-to-end through the host-buffer ABI: ordinary (pageable) host arrays, as a
    # drop-in caller passes them; with pinned arrays beside it where the workload has both
    def e2e_time(step):
        step()
        barrier()
        ts = []
        for _ in range(max(3, args.steps // 2)):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            step()
            ts.append((time.perf_counter() - t0) * 1e3)
        ms = float(np.median(ts))
        return max_over_ranks(ms, "cuda") if world > 1 else ms
    e2e_step_ms = e2e_time(wl.e2e_step)
    if hasattr(wl, "e2e_step_pinned"):
        pinned_ms = e2e_time(wl.e2e_step_pinned)
        extra["e2e_pinned_host_buffers"] = {"value": world * wl.batch / (pinned_ms * 1e-3), "unit": UNIT}

    # roofline of the dominant kernel
    mean_ms = {name: float(np.mean(v)) for name, v in times.items()}
    dom = max(mean_ms, key=mean_ms.get)
    dom_bytes, dom_ops = wl.roofline_inputs(dom)
    peak, peak_kind = _peaks()
    dom_ms = mean_ms[dom]
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    # compute roof: the CUDA-core pipe, one scalar op per lane per clock (the sweeps
    # round each + and * separately, -fmad=false); flops per unit by value kind
    # (echidna_b200.opcost), libm calls not counted
    from echidna_b200 import opcost
    sm_mhz = 1965.0
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            sm_mhz = float(json.load(f).get("sm_max_mhz", sm_mhz))
    except OSError:
        pass
    pipe_ops = opcost.pipe_peak_ops(wl.describe()[1] == "f64", sm_mhz)
    pipe_peak = pipe_ops / 1e12
    combined = opcost.roofline(dom_bytes, dom_ops, dom_ms * 1e-3, peak, pipe_ops)
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(f"{wl.name}:{dom}")

    cfg, dtype = wl.describe()
    cfg.update({"l2": "flushed between steps (256 MiB write outside the events)",
                "parallelism": f"points sharded, {world} rank(s)"})
    h2d, d2h = wl.io_bytes()
    line = {
        "metric": METRIC, "value": world * wl.batch / (step_ms * 1e-3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic", "config": cfg,
        "gpu_launches": wl.launches_per_step * args.steps,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": dom_bytes, "launch_ms": dom_ms,
                     "scalar_ops_per_launch": dom_ops, "scalar_tops": dom_ops / (dom_ms * 1e-3) / 1e12,
                     "scalar_pipe_peak_tops": pipe_peak, "scalar_pipe_frac": dom_ops / (dom_ms * 1e-3) / 1e12 / pipe_peak,
                     "scalar_pipe_peak_source": "nominal: 148 SMs x 128 FP32 lanes x max SM clock "
                                                "(FP64: x 1/2); one op per lane per clock, no FMA",
                     "t_roof": combined},
        "e2e": {"value": world * wl.batch / (e2e_step_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "clocks": clk.summary(),
        "detail": {**{f"{k} ms": v for k, v in mean_ms.items()}, **wl.detail(), **extra},
    }
    if rank == 0 and not args.no_cpu_baseline:
        nth = os.cpu_count() or 1
        v, sample = wl.cpu_reference(10.0, nth)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": nth, "kind": "port", "sample": sample,
                                "cpu_model": _cpu_model()}
        v1, sample1 = wl.cpu_reference(3.0, 1)
        line["cpu_baseline"]["single_thread"] = {"value": v1, "sample": sample1}
        if hasattr(wl, "accuracy"):
            line["detail"]["accuracy_256_points"] = wl.accuracy(256)
        if dtype == "f32" and "dtype" in wl.cpu_reference.__code__.co_varnames:
            # the same CPU path in FP32, so the FP32 GPU figure has a same-precision CPU number beside it
            v32, sample32 = wl.cpu_reference(5.0, nth, dtype=np.float32)
            line["cpu_baseline"]["same_precision_f32"] = {"value": v32, "sample": sample32}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del kernels, wl
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
