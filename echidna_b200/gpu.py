"""Host-side mirror of echidna's CUDA backend API, over the engine's C ABI.

Names, argument meaning and error behaviour follow ``src/gpu/mod.rs`` and
``src/gpu/cuda_backend.rs``:

* ``CudaContext.new()`` returns ``None`` without a device (``cuda_backend.rs:503-552``).
* ``upload_tape(GpuTapeData)`` raises ``TapeUploadPanic`` for invalid data, where the
  Rust method panics (``cuda_backend.rs:628-631``); ``upload_tape_f64`` raises
  ``GpuError`` (``cuda_backend.rs:566-611``).
* Batch calls raise ``GpuError`` for the ``Err`` results of the reference (for
  example ``"batch_size must be non-zero"``) and ``AssertionError`` for the length
  mismatches the reference asserts on.

All work runs in the CUDA library; nothing here computes derivatives.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _lib
from .tape import BytecodeTape, OpCode


class GpuError(Exception):
    """``GpuError`` (``src/gpu/mod.rs:276-301``)."""

    kind = "Other"

    def __init__(self, msg: str = ""):
        super().__init__(msg)
        self.msg = msg


class NoDevice(GpuError):
    kind = "NoDevice"


class ShaderCompilation(GpuError):
    kind = "ShaderCompilation"


class OutOfMemory(GpuError):
    kind = "OutOfMemory"


class CustomOpsNotSupported(GpuError):
    kind = "CustomOpsNotSupported"


class DeviceTimeout(GpuError):
    kind = "Timeout"


class TapeUploadPanic(RuntimeError):
    """The reference panics here; the message starts with ``refusing to upload``."""


def _raise(status: int):
    msg = _lib.last_error()
    if status == _lib.INVALID_ARG:
        raise AssertionError(msg)
    cls = {
        _lib.NO_DEVICE: NoDevice,
        _lib.SHADER_COMPILATION: ShaderCompilation,
        _lib.OUT_OF_MEMORY: OutOfMemory,
        _lib.CUSTOM_OPS_NOT_SUPPORTED: CustomOpsNotSupported,
        _lib.TIMEOUT: DeviceTimeout,
    }.get(status, GpuError)
    raise cls(msg)


def _check(status: int):
    if status != _lib.OK:
        _raise(status)


# WGPU_MAX_BUFFER_BYTES (src/gpu/mod.rs:619): the default chunk budget of the chunked Taylor call.
WGPU_MAX_BUFFER_BYTES = 128 * 1024 * 1024


@dataclass
class GpuTapeData:
    """Flattened tape for upload (``src/gpu/mod.rs:313-334``), f32 constants."""

    opcodes: np.ndarray
    arg0: np.ndarray
    arg1: np.ndarray
    constants: np.ndarray
    num_ops: int
    num_inputs: int
    num_variables: int
    output_index: int
    output_indices: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.uint32))

    @classmethod
    def _build(cls, tape: BytecodeTape, constants: np.ndarray) -> "GpuTapeData":
        op, a0, a1, _ = tape.arrays()
        n = len(op)
        return cls(op, a0, a1, np.ascontiguousarray(constants, dtype=np.float32), n, tape.num_inputs, n,
                   tape.output_index, np.asarray(tape.all_output_indices(), dtype=np.uint32))

    @classmethod
    def from_tape(cls, tape: BytecodeTape) -> "GpuTapeData":
        """``GpuTapeData::from_tape`` (``src/gpu/mod.rs:365-371``)."""
        if tape.has_custom_ops:
            raise CustomOpsNotSupported("tape contains custom ops which cannot run on GPU")
        return cls._build(tape, np.asarray(tape.values, dtype=np.float32))

    @classmethod
    def from_tape_f64_lossy(cls, tape: BytecodeTape) -> "GpuTapeData":
        """``GpuTapeData::from_tape_f64_lossy`` (``src/gpu/mod.rs:378-384``)."""
        if tape.has_custom_ops:
            raise CustomOpsNotSupported("tape contains custom ops which cannot run on GPU")
        # `as f32` in the reference: magnitudes past f32's range become +-inf
        with np.errstate(over="ignore"):
            vals = np.asarray(tape.values, dtype=np.float64).astype(np.float32)
        return cls._build(tape, vals)

    def _arrays(self):
        return (np.ascontiguousarray(self.opcodes, dtype=np.uint32), np.ascontiguousarray(self.arg0, dtype=np.uint32),
                np.ascontiguousarray(self.arg1, dtype=np.uint32),
                np.ascontiguousarray(self.constants, dtype=np.float32),
                np.ascontiguousarray(self.output_indices, dtype=np.uint32))

    def validate(self) -> None:
        """``GpuTapeData::validate`` (``src/gpu/mod.rs:397-564``); raises ``GpuError``."""
        lib = _lib.load()
        op, a0, a1, c, outs = self._arrays()
        st = lib.ech_validate_gpu_tape_data(_lib.ptr(op), len(op), _lib.ptr(a0), len(a0), _lib.ptr(a1), len(a1),
                                            len(c), self.num_ops, self.num_inputs, self.num_variables,
                                            self.output_index, _lib.ptr(outs), len(outs))
        _check(st)


@dataclass
class TaylorBatchResult:
    """``TaylorBatchResult`` (``src/gpu/mod.rs:227-240``)."""

    values: np.ndarray
    c1s: np.ndarray
    c2s: np.ndarray


@dataclass
class TaylorKthBatchResult:
    """``TaylorKthBatchResult`` (``src/gpu/mod.rs:261-272``)."""

    coefficients: List[np.ndarray]
    order: int


@dataclass
class EstimatorResult:
    """``EstimatorResult`` (``src/stde/types.rs:9-22``)."""

    value: float
    estimate: float
    sample_variance: float
    standard_error: float
    num_samples: int


class _TapeHandle:
    def __init__(self, ctx: "CudaContext", handle: int, f64: bool):
        self._ctx = ctx
        self._h = ctypes.c_void_p(handle)
        self.f64 = f64
        lib = _lib.load()
        self.num_outputs = int(lib.ech_tape_num_outputs(self._h))
        self.num_inputs = int(lib.ech_tape_num_inputs(self._h))
        self.num_variables = int(lib.ech_tape_num_variables(self._h))

    def __del__(self):
        try:
            if self._h:
                _lib.load().ech_tape_destroy(self._h)
                self._h = None
        except Exception:
            pass


class CudaTapeBuffers(_TapeHandle):
    """Uploaded tape with f32 constants (``src/gpu/cuda_backend.rs:449-459``)."""


class CudaTapeBuffersF64(_TapeHandle):
    """Uploaded tape with f64 constants (``src/gpu/cuda_backend.rs:462-472``)."""


def _arr(x, dt):
    return np.ascontiguousarray(np.asarray(x, dtype=dt).ravel())


class CudaContext:
    """B200 engine context: same methods as echidna's ``CudaContext``."""

    def __init__(self, handle):
        self._h = handle
        self._children = []  # handles that must be released before the context

    @staticmethod
    def new(device: int = 0) -> Optional["CudaContext"]:
        lib = _lib.load()
        h = ctypes.c_void_p()
        st = lib.ech_ctx_create(device, ctypes.byref(h))
        if st != _lib.OK:
            return None
        return CudaContext(h)

    def close(self):
        for c in getattr(self, "_children", []):
            c.close()
        self._children = []
        if getattr(self, "_h", None):
            _lib.load().ech_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- tuning ---------------------------------------------------------------
    def set_launch(self, threads: int = 0, points_per_thread: int = 0, smem_reg_cap: int = 0):
        _check(_lib.load().ech_ctx_set_launch(self._h, threads, points_per_thread, smem_reg_cap))

    def set_dense_kernel(self, always: bool = True):
        """Run every sweep on the kernel build with the dense-group executor, on the fixed
        launch shape (``ech_ctx_set_dense_kernel``); ``False`` restores the automatic choice."""
        _check(_lib.load().ech_ctx_set_dense_kernel(self._h, 1 if always else 0))

    FP32_COMPENSATED_JETS, FP32_COMPENSATED_MEANS, FP32_PLAIN_MEANS = 1, 2, 4

    def set_fp32_mode(self, flags: int = 0):
        """FP32 options of the batch STDE calls (``ech_ctx_set_fp32_mode``): compensated
        linear chains in the jet sweep, and FP32 compensated or plain per-point means
        instead of the FP64 Welford reduction."""
        _check(_lib.load().ech_ctx_set_fp32_mode(self._h, int(flags)))

    def set_autotune(self, enable: bool):
        _check(_lib.load().ech_ctx_set_autotune(self._h, 1 if enable else 0))

    def launch_shape(self, tape: _TapeHandle, kind: str, n_units: int, order: int = 0) -> dict:
        kinds = {"forward": 0, "gradient": 1, "hvp": 2, "tangent": 3, "taylor": 4}
        buf = (ctypes.c_uint64 * 8)()
        _check(_lib.load().ech_tape_launch_shape(self._h, tape._h, kinds[kind], order, n_units, buf))
        keys = ["threads", "points_per_thread", "ctas_per_sm", "smem_reg_cap", "smem_regs", "far_slots",
                "traj_slots", "tuned"]
        d = dict(zip(keys, [int(v) for v in buf]))
        d["dense_kernel"] = (d["tuned"] >> 1) & 1   # the tuner chose the dense-group kernel build
        d["tuned"] &= 1
        return d

    def program_stats(self, tape: _TapeHandle, kind: str, n_units: int, order: int = 0) -> dict:
        """The encoded device program a sweep of ``n_units`` runs (``ech_tape_program_stats``)."""
        kinds = {"forward": 0, "gradient": 1, "hvp": 2, "tangent": 3, "taylor": 4, "taylor_direct": 5}
        buf = (ctypes.c_uint64 * 5)()
        _check(_lib.load().ech_tape_program_stats(self._h, tape._h, kinds[kind], order, n_units, buf))
        keys = ["fwd_records", "rev_records", "dense_groups", "gather_tiles", "dense_kernel"]
        return dict(zip(keys, [int(v) for v in buf]))

    def plan_stats(self, tape: _TapeHandle, kind: str, order: int = 0) -> dict:
        kinds = {"forward": 0, "gradient": 1, "hvp": 2, "tangent": 3, "taylor": 4, "taylor_direct": 5}
        buf = (ctypes.c_uint64 * 12)()
        _check(_lib.load().ech_tape_plan_stats(self._h, tape._h, kinds[kind], order, int(tape.f64), buf))
        keys = ["fwd_ops", "rev_ops", "max_live_fwd", "max_live_rev", "traj_values", "flops_fwd", "flops_rev",
                "specials_fwd", "specials_rev", "smem_regs", "far_slots", "n_instructions"]
        return dict(zip(keys, [int(v) for v in buf]))

    # -- upload ---------------------------------------------------------------
    def upload_tape(self, data: GpuTapeData) -> CudaTapeBuffers:
        lib = _lib.load()
        op, a0, a1, c, outs = data._arrays()
        h = ctypes.c_void_p()
        st = lib.ech_upload_tape_f32(self._h, _lib.ptr(op), len(op), _lib.ptr(a0), len(a0), _lib.ptr(a1), len(a1),
                                     _lib.ptr(c), len(c), data.num_ops, data.num_inputs, data.num_variables,
                                     data.output_index, _lib.ptr(outs), len(outs), ctypes.byref(h))
        if st != _lib.OK:
            raise TapeUploadPanic(_lib.last_error())
        return CudaTapeBuffers(self, h.value, False)

    def upload_tape_f64(self, tape: BytecodeTape) -> CudaTapeBuffersF64:
        lib = _lib.load()
        op, a0, a1, vals = tape.arrays()
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        outs = np.asarray(tape.output_indices, dtype=np.uint32)
        h = ctypes.c_void_p()
        st = lib.ech_upload_tape_f64(self._h, _lib.ptr(op), _lib.ptr(a0), _lib.ptr(a1), _lib.ptr(vals), len(op),
                                     tape.num_inputs, tape.output_index, _lib.ptr(outs), len(outs),
                                     1 if tape.has_custom_ops else 0, ctypes.byref(h))
        _check(st)
        return CudaTapeBuffersF64(self, h.value, True)

    def num_outputs(self, tape: _TapeHandle) -> int:
        return tape.num_outputs

    # -- sweeps ---------------------------------------------------------------
    def _forward(self, tape, inputs, batch_size, dt, fn):
        x = _arr(inputs, dt)
        out = np.empty(int(batch_size) * tape.num_outputs, dtype=dt)
        _check(fn(self._h, tape._h, _lib.ptr(x), x.size, batch_size, _lib.ptr(out), out.size))
        return out

    def forward_batch(self, tape: CudaTapeBuffers, inputs, batch_size: int) -> np.ndarray:
        return self._forward(tape, inputs, batch_size, np.float32, _lib.load().ech_forward_batch_f32)

    def forward_batch_f64(self, tape: CudaTapeBuffersF64, inputs, batch_size: int) -> np.ndarray:
        return self._forward(tape, inputs, batch_size, np.float64, _lib.load().ech_forward_batch_f64)

    def _gradient(self, tape, inputs, batch_size, dt, fn):
        x = _arr(inputs, dt)
        out = np.empty(int(batch_size) * tape.num_outputs, dtype=dt)
        g = np.empty(int(batch_size) * tape.num_inputs, dtype=dt)
        _check(fn(self._h, tape._h, _lib.ptr(x), x.size, batch_size, _lib.ptr(out), out.size, _lib.ptr(g), g.size))
        return out, g

    def gradient_batch(self, tape: CudaTapeBuffers, inputs, batch_size: int):
        return self._gradient(tape, inputs, batch_size, np.float32, _lib.load().ech_gradient_batch_f32)

    def gradient_batch_f64(self, tape: CudaTapeBuffersF64, inputs, batch_size: int):
        return self._gradient(tape, inputs, batch_size, np.float64, _lib.load().ech_gradient_batch_f64)

    def _hvp(self, tape, x, dirs, batch_size, dt, fn):
        x = _arr(x, dt)
        d = _arr(dirs, dt)
        g = np.empty(int(batch_size) * tape.num_inputs, dtype=dt)
        h = np.empty(int(batch_size) * tape.num_inputs, dtype=dt)
        _check(fn(self._h, tape._h, _lib.ptr(x), x.size, _lib.ptr(d), d.size, batch_size, _lib.ptr(g), g.size,
                  _lib.ptr(h), h.size))
        return g, h

    def hvp_batch(self, tape: CudaTapeBuffers, x, tangent_dirs, batch_size: int):
        return self._hvp(tape, x, tangent_dirs, batch_size, np.float32, _lib.load().ech_hvp_batch_f32)

    def hvp_batch_f64(self, tape: CudaTapeBuffersF64, x, tangent_dirs, batch_size: int):
        return self._hvp(tape, x, tangent_dirs, batch_size, np.float64, _lib.load().ech_hvp_batch_f64)

    def hvp_batch_points(self, tape: CudaTapeBuffers, xs, tangent_dirs, batch_size: int):
        """Extension: per-point HVP ``(grad f(x_b), H(x_b) v_b)``."""
        return self._hvp(tape, xs, tangent_dirs, batch_size, np.float32, _lib.load().ech_hvp_batch_points_f32)

    def hvp_batch_points_f64(self, tape: CudaTapeBuffersF64, xs, tangent_dirs, batch_size: int):
        return self._hvp(tape, xs, tangent_dirs, batch_size, np.float64, _lib.load().ech_hvp_batch_points_f64)

    def _tangent(self, tape, primals, seeds, batch_size, dt, fn):
        p = _arr(primals, dt)
        s = _arr(seeds, dt)
        v = np.empty(int(batch_size) * tape.num_outputs, dtype=dt)
        t = np.empty(int(batch_size) * tape.num_outputs, dtype=dt)
        _check(fn(self._h, tape._h, _lib.ptr(p), p.size, _lib.ptr(s), s.size, batch_size, _lib.ptr(v), _lib.ptr(t),
                  v.size))
        return v, t

    def tangent_forward_batch(self, tape: CudaTapeBuffers, primals, seeds, batch_size: int):
        """The reference's ``tangent_forward`` kernel (JVP per row): ``(values, tangents)``."""
        return self._tangent(tape, primals, seeds, batch_size, np.float32, _lib.load().ech_tangent_forward_batch_f32)

    def tangent_forward_batch_f64(self, tape: CudaTapeBuffersF64, primals, seeds, batch_size: int):
        return self._tangent(tape, primals, seeds, batch_size, np.float64, _lib.load().ech_tangent_forward_batch_f64)

    def _taylor(self, tape, primals, seeds, batch_size, order, dt, fn):
        p = _arr(primals, dt)
        s = _arr(seeds, dt)
        total = int(batch_size) * tape.num_outputs
        c = np.empty(max(int(order), 1) * total, dtype=dt)
        _check(fn(self._h, tape._h, _lib.ptr(p), p.size, _lib.ptr(s), s.size, batch_size, int(order), _lib.ptr(c),
                  int(order) * total))
        return TaylorKthBatchResult([c[k * total:(k + 1) * total] for k in range(int(order))], int(order))

    def taylor_forward_kth_batch(self, tape: CudaTapeBuffers, primal_inputs, direction_seeds, batch_size: int,
                                 order: int) -> TaylorKthBatchResult:
        return self._taylor(tape, primal_inputs, direction_seeds, batch_size, order, np.float32,
                            _lib.load().ech_taylor_forward_kth_batch_f32)

    def taylor_forward_kth_batch_f64(self, tape: CudaTapeBuffersF64, primal_inputs, direction_seeds, batch_size: int,
                                     order: int) -> TaylorKthBatchResult:
        return self._taylor(tape, primal_inputs, direction_seeds, batch_size, order, np.float64,
                            _lib.load().ech_taylor_forward_kth_batch_f64)

    def taylor_forward_2nd_batch(self, tape: CudaTapeBuffers, primal_inputs, direction_seeds,
                                 batch_size: int) -> TaylorBatchResult:
        """Default trait method: ``taylor_forward_kth_batch(order=3)`` (``src/gpu/mod.rs:189-204``)."""
        k = self.taylor_forward_kth_batch(tape, primal_inputs, direction_seeds, batch_size, 3)
        return TaylorBatchResult(*k.coefficients)

    def taylor_forward_2nd_batch_f64(self, tape: CudaTapeBuffersF64, primal_inputs, direction_seeds,
                                     batch_size: int) -> TaylorBatchResult:
        k = self.taylor_forward_kth_batch_f64(tape, primal_inputs, direction_seeds, batch_size, 3)
        return TaylorBatchResult(*k.coefficients)

    def taylor_forward_2nd_batch_chunked(self, tape: CudaTapeBuffers, primal_inputs, direction_seeds,
                                         batch_size: int, num_inputs: int, num_variables: int,
                                         max_buffer_bytes: int = WGPU_MAX_BUFFER_BYTES) -> TaylorBatchResult:
        """``taylor_forward_2nd_batch_chunked`` (``src/gpu/mod.rs:652-733``): the same chunk
        size rule (jets working buffer of ``num_variables * 3 * 4`` bytes per element, the
        65535 x 256 dispatch cap and the u32 index cap), each chunk one K=3 sweep."""
        if batch_size == 0:
            e = np.zeros(0, np.float32)
            return TaylorBatchResult(e, e.copy(), e.copy())
        per = int(num_variables) * 3 * 4
        if per == 0:
            raise GpuError("num_variables is zero")
        chunk = int(max_buffer_bytes) // per
        if chunk == 0:
            raise GpuError(f"max_buffer_bytes ({max_buffer_bytes}) too small for a single element "
                           f"({per} bytes per element)")
        chunk = min(chunk, 65535 * 256, 0xFFFFFFFF // (int(num_variables) * 3))
        p = _arr(primal_inputs, np.float32)
        s = _arr(direction_seeds, np.float32)
        if batch_size <= chunk:
            return self.taylor_forward_2nd_batch(tape, p, s, batch_size)
        ni = int(num_inputs)
        vals, c1s, c2s = [], [], []
        off = 0
        while off < batch_size:
            n = min(chunk, batch_size - off)
            r = self.taylor_forward_2nd_batch(tape, p[off * ni:(off + n) * ni], s[off * ni:(off + n) * ni], n)
            vals.append(r.values)
            c1s.append(r.c1s)
            c2s.append(r.c2s)
            off += n
        return TaylorBatchResult(np.concatenate(vals), np.concatenate(c1s), np.concatenate(c2s))

    # -- sparse drop-ins (src/gpu/cuda_backend.rs:306-441) ---------------------
    def sparse_jacobian(self, tape: CudaTapeBuffers, tape_cpu: BytecodeTape, x):
        from .sparse import sparse_jacobian_gpu
        return sparse_jacobian_gpu(self, tape, tape_cpu, x, np.float32)

    def sparse_jacobian_f64(self, tape: CudaTapeBuffersF64, tape_cpu: BytecodeTape, x):
        from .sparse import sparse_jacobian_gpu
        return sparse_jacobian_gpu(self, tape, tape_cpu, x, np.float64)

    def sparse_hessian(self, tape: CudaTapeBuffers, tape_cpu: BytecodeTape, x):
        from .sparse import sparse_hessian_gpu
        return sparse_hessian_gpu(self, tape, tape_cpu, x, np.float32)

    def sparse_hessian_f64(self, tape: CudaTapeBuffersF64, tape_cpu: BytecodeTape, x):
        from .sparse import sparse_hessian_gpu
        return sparse_hessian_gpu(self, tape, tape_cpu, x, np.float64)


class _MultiItem(ctypes.Structure):
    _fields_ = [("tape", ctypes.c_void_p), ("xs", ctypes.c_void_p), ("dirs", ctypes.c_void_p),
                ("n_points", ctypes.c_uint32), ("pad", ctypes.c_uint32), ("grads", ctypes.c_void_p),
                ("hvps", ctypes.c_void_p)]


class MultiTapeHvp:
    """Gradient + per-point HVP of many tapes in one persistent launch (extension).

    ``items``: sequence of ``(tape, xs_ptr, dirs_ptr, n_points, grads_ptr, hvps_ptr)``
    with device pointers (``[n_points][num_inputs]`` each).  The buffers are bound
    to the launch; ``launch(stream)`` enqueues it without synchronising, so it can
    be captured in a CUDA graph once created.
    """

    def __init__(self, ctx: "CudaContext", items, f64: bool = False, autotune: bool = True):
        lib = _lib.load()
        arr = (_MultiItem * len(items))()
        for k, (tape, xs, dirs, n, g, h) in enumerate(items):
            arr[k] = _MultiItem(tape._h, xs, dirs, int(n), 0, g, h)
        self._items = arr
        self._tapes = [it[0] for it in items]
        self._ctx = ctx
        h = ctypes.c_void_p()
        _check(lib.ech_multi_create(ctx._h, 1 if f64 else 0, ctypes.cast(arr, ctypes.c_void_p), len(items),
                                    1 if autotune else 0, ctypes.byref(h)))
        self._h = h
        ctx._children.append(self)

    def launch(self, stream: int = 0):
        _check(_lib.load().ech_multi_launch(self._h, ctypes.c_void_p(stream)))

    def info(self) -> dict:
        buf = (ctypes.c_uint64 * 9)()
        _check(_lib.load().ech_multi_info(self._h, buf))
        keys = ["threads", "points_per_thread", "ctas_per_sm", "smem_reg_cap", "grid", "tiles", "jobs",
                "scratch_bytes_per_cta", "tuned"]
        d = dict(zip(keys, [int(v) for v in buf]))
        d["dense_kernel"] = (d["tuned"] >> 1) & 1
        d["tuned"] &= 1
        return d

    def close(self):
        if getattr(self, "_h", None) and getattr(self._ctx, "_h", None):
            _lib.load().ech_multi_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
