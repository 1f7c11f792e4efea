"""ctypes binding of ``libechidna_b200.so`` (the C ABI in ``include/echidna_b200.h``).

The library is the product path: there is no fallback.  If the shared object is
missing or fails to load, every entry point raises ``EngineNotBuilt``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# ECHIDNA_B200_VARIANT=bounds selects the device bounds-checked build of the same engine
LIB_PATH = os.path.join(_HERE, "libechidna_b200_bounds.so" if os.environ.get("ECHIDNA_B200_VARIANT") == "bounds"
                        else "libechidna_b200.so")


class EngineNotBuilt(RuntimeError):
    """The CUDA engine library is not built or cannot be loaded."""


# ech_status codes
OK, NO_DEVICE, SHADER_COMPILATION, OUT_OF_MEMORY, CUSTOM_OPS_NOT_SUPPORTED, OTHER, TIMEOUT, INVALID_ARG = range(8)


class EstimatorResultC(ctypes.Structure):
    _fields_ = [
        ("value", ctypes.c_double),
        ("estimate", ctypes.c_double),
        ("sample_variance", ctypes.c_double),
        ("standard_error", ctypes.c_double),
        ("num_samples", ctypes.c_uint64),
    ]


_lib = None
_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_SZ = ctypes.c_size_t
_I = ctypes.c_int

_SIGS = {
    "ech_last_error": ([], ctypes.c_char_p),
    "ech_version": ([], ctypes.c_char_p),
    "ech_ctx_create": ([_I, ctypes.POINTER(_P)], _I),
    "ech_ctx_destroy": ([_P], None),
    "ech_ctx_set_launch": ([_P, _U32, _U32, _U32], _I),
    "ech_ctx_synchronize": ([_P], _I),
    "ech_validate_bytecode_tape": ([_P, _P, _P, _U32, _U32, _U32, _P, _U32, _I], _I),
    "ech_validate_gpu_tape_data": ([_P, _U32, _P, _U32, _P, _U32, _U32, _U32, _U32, _U32, _U32, _P, _U32], _I),
    "ech_upload_tape_f32": ([_P, _P, _U32, _P, _U32, _P, _U32, _P, _U32, _U32, _U32, _U32, _U32, _P, _U32,
                             ctypes.POINTER(_P)], _I),
    "ech_upload_tape_f64": ([_P, _P, _P, _P, _P, _U32, _U32, _U32, _P, _U32, _I, ctypes.POINTER(_P)], _I),
    "ech_tape_destroy": ([_P], None),
    "ech_tape_num_outputs": ([_P], _U32),
    "ech_tape_num_inputs": ([_P], _U32),
    "ech_tape_num_variables": ([_P], _U32),
    "ech_forward_batch_f32": ([_P, _P, _P, _SZ, _U32, _P, _SZ], _I),
    "ech_forward_batch_f64": ([_P, _P, _P, _SZ, _U32, _P, _SZ], _I),
    "ech_gradient_batch_f32": ([_P, _P, _P, _SZ, _U32, _P, _SZ, _P, _SZ], _I),
    "ech_gradient_batch_f64": ([_P, _P, _P, _SZ, _U32, _P, _SZ, _P, _SZ], _I),
    "ech_hvp_batch_f32": ([_P, _P, _P, _SZ, _P, _SZ, _U32, _P, _SZ, _P, _SZ], _I),
    "ech_hvp_batch_f64": ([_P, _P, _P, _SZ, _P, _SZ, _U32, _P, _SZ, _P, _SZ], _I),
    "ech_hvp_batch_points_f32": ([_P, _P, _P, _SZ, _P, _SZ, _U32, _P, _SZ, _P, _SZ], _I),
    "ech_hvp_batch_points_f64": ([_P, _P, _P, _SZ, _P, _SZ, _U32, _P, _SZ, _P, _SZ], _I),
    "ech_tangent_forward_batch_f32": ([_P, _P, _P, _SZ, _P, _SZ, _U32, _P, _P, _SZ], _I),
    "ech_tangent_forward_batch_f64": ([_P, _P, _P, _SZ, _P, _SZ, _U32, _P, _P, _SZ], _I),
    "ech_taylor_forward_kth_batch_f32": ([_P, _P, _P, _SZ, _P, _SZ, _U32, _U32, _P, _SZ], _I),
    "ech_taylor_forward_kth_batch_f64": ([_P, _P, _P, _SZ, _P, _SZ, _U32, _U32, _P, _SZ], _I),
    "ech_laplacian_gpu_f32": ([_P, _P, _P, _SZ, _P, _U32, _P], _I),
    "ech_hessian_diagonal_gpu_f32": ([_P, _P, _P, _SZ, _P, _P], _I),
    "ech_laplacian_with_control_gpu_f32": ([_P, _P, _P, _SZ, _P, _U32, _P, _P], _I),
    "ech_laplacian_batch_f32": ([_P, _P, _P, _SZ, _U32, _P, _SZ, _U32, _I, _U64, _P], _I),
    "ech_laplacian_batch_f64": ([_P, _P, _P, _SZ, _U32, _P, _SZ, _U32, _I, _U64, _P], _I),
    "ech_forward_batch_device": ([_P, _P, _I, _P, _U32, _P, _P], _I),
    "ech_gradient_batch_device": ([_P, _P, _I, _P, _U32, _P, _P, _P], _I),
    "ech_hvp_batch_device": ([_P, _P, _I, _P, _I, _P, _U32, _P, _P, _P], _I),
    "ech_taylor_batch_device": ([_P, _P, _I, _P, _P, _U32, _U32, _P, _P], _I),
    "ech_noalloc_region_bytes": ([], _SZ),
    "ech_grad_checkpointed_device": ([_P, _P, _P, _I, _P, _U32, _U32, _U32, _P], _I),
    "ech_laplacian_hutchpp_f32": ([_P, _P, _P, _SZ, _P, _U32, _P, _U32, _P], _I),
    "ech_parabolic_diffusion_f32": ([_P, _P, _P, _SZ, _P, _U32, _P, _P], _I),
    "ech_parabolic_diffusion_stochastic_f32": ([_P, _P, _P, _SZ, _P, _U32, _P, _U32, _P], _I),
    "ech_dense_stde_2nd_f32": ([_P, _P, _P, _SZ, _P, _P, _U32, _P], _I),
    "ech_divergence_f32": ([_P, _P, _P, _SZ, _P, _U32, _P, _P], _I),
    "ech_laplacian_hutchpp_f64": ([_P, _P, _P, _SZ, _P, _U32, _P, _U32, _P], _I),
    "ech_parabolic_diffusion_f64": ([_P, _P, _P, _SZ, _P, _U32, _P, _P], _I),
    "ech_parabolic_diffusion_stochastic_f64": ([_P, _P, _P, _SZ, _P, _U32, _P, _U32, _P], _I),
    "ech_dense_stde_2nd_f64": ([_P, _P, _P, _SZ, _P, _P, _U32, _P], _I),
    "ech_divergence_f64": ([_P, _P, _P, _SZ, _P, _U32, _P, _P], _I),
    "ech_hessian_diagonal_batch_device": ([_P, _P, _I, _P, _U32, _P, _P], _I),
    "ech_sparse_trace_batch_device": ([_P, _P, _I, _P, _U32, _P, _U32, _U64, _P, _P], _I),
    "ech_gemm_bf16": ([_P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P], _I),
    "ech_mlp_create": ([_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P], _I),
    "ech_mlp_train_step": ([_P, _P, _P, _I, ctypes.c_float, _P], _I),
    "ech_mlp_forward": ([_P, _P, _I, _P, _P], _I),
    "ech_mlp_gradients": ([_P, _P, _P, _I, _P, _P, _P, _P, _P, _P, _P], _I),
    "ech_ctx_set_fp32_mode": ([_P, _U32], _I),
    "ech_ctx_set_dense_kernel": ([_P, _I], _I),
    "ech_tape_program_stats": ([_P, _P, _I, _U32, _U64, _P], _I),
    "ech_mlp_get_weights": ([_P, _P, _P, _P, _P, _P, _P], _I),
    "ech_mlp_destroy": ([_P], None),
    "ech_multi_create": ([_P, _I, _P, _U32, _I, _P], _I),
    "ech_multi_launch": ([_P, _P], _I),
    "ech_multi_info": ([_P, ctypes.POINTER(_U64)], _I),
    "ech_multi_destroy": ([_P], None),
    "ech_laplacian_batch_device": ([_P, _P, _I, _P, _U32, _P, _U32, _I, _U64, _P, _P], _I),
    "ech_diagonal_kth_order_stochastic_f32": ([_P, _P, _P, _SZ, _U32, _P, _SZ, _P], _I),
    "ech_diagonal_kth_order_stochastic_f64": ([_P, _P, _P, _SZ, _U32, _P, _SZ, _P], _I),
    "ech_diagonal_kth_order_f32": ([_P, _P, _P, _SZ, _U32, _P, _P], _I),
    "ech_diagonal_kth_order_f64": ([_P, _P, _P, _SZ, _U32, _P, _P], _I),
    "ech_estimate_f32": ([_P, _P, _P, _SZ, _I, _P, _U32, _P, _P], _I),
    "ech_estimate_f64": ([_P, _P, _P, _SZ, _I, _P, _U32, _P, _P], _I),
    "ech_stde_sparse_batch_f32": ([_P, _P, _P, _SZ, _U32, _U32, _P, _P, _P, _P, _P, _P, _P, ctypes.c_float, _P, _U32,
                                   _P], _I),
    "ech_stde_sparse_batch_f64": ([_P, _P, _P, _SZ, _U32, _U32, _P, _P, _P, _P, _P, _P, _P, ctypes.c_double, _P, _U32,
                                   _P], _I),
    "ech_detect_hessian_sparsity": ([_P, _P, _P, _U32, _U32, _P, _P, _SZ, ctypes.POINTER(_SZ)], _I),
    "ech_detect_jacobian_sparsity": ([_P, _P, _P, _U32, _U32, _P, _U32, _P, _P, _SZ, ctypes.POINTER(_SZ)], _I),
    "ech_greedy_coloring": ([_U32, _P, _P, _SZ, _P, ctypes.POINTER(_U32)], _I),
    "ech_column_coloring": ([_U32, _U32, _P, _P, _SZ, _P, ctypes.POINTER(_U32)], _I),
    "ech_row_coloring": ([_U32, _U32, _P, _P, _SZ, _P, ctypes.POINTER(_U32)], _I),
    "ech_ctx_set_autotune": ([_P, _I], _I),
    "ech_tape_launch_shape": ([_P, _P, _I, _U32, _U64, ctypes.POINTER(_U64)], _I),
    "ech_gradient_batch_device_noalloc": ([_P, _P, _I, _P, _U32, _P, _P, _P], _I),
    "ech_tape_plan_stats": ([_P, _P, _I, _U32, _I, ctypes.POINTER(_U64)], _I),
    "ech_plan_dump": ([_P, _P, _P, _P, _U32, _U32, _U32, _P, _U32, _I, _U32, _P, _SZ, _P, _SZ, _P, _SZ, _P, _SZ,
                       _P, _SZ, _P, _SZ, _U32, ctypes.POINTER(_U64)], _I),
}


def load():
    """Loads the library (once).  Raises ``EngineNotBuilt`` if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise EngineNotBuilt(
            f"{LIB_PATH} is missing; build it with `python -m echidna_b200.build` "
            "(the engine has no CPU fallback)")
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as e:  # pragma: no cover
        raise EngineNotBuilt(f"cannot load {LIB_PATH}: {e}") from e
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def exported_symbols():
    return sorted(_SIGS)


def last_error() -> str:
    return load().ech_last_error().decode()


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def validate_bytecode_tape(op, a0, a1, nv, ni, output_index, outs, has_custom):
    """Returns None when valid, else the reference's error message."""
    lib = load()
    st = lib.ech_validate_bytecode_tape(ptr(op), ptr(a0), ptr(a1), nv, ni, output_index, ptr(outs), len(outs),
                                        has_custom)
    if st == OK:
        return None
    return last_error()
