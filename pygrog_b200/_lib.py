"""ctypes binding of ``libpygrog_b200.so`` (the C ABI in ``include/pygrog_b200.h``).

There is no fallback: if the library is missing or no CUDA device is
present, every operation raises.  Tensors are passed as raw device pointers;
kernels are launched on torch's current CUDA stream.
"""

from __future__ import annotations

import ctypes
import os
import pathlib

import torch

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "_lib" / "libpygrog_b200.so"

PGB_C64 = 0
PGB_C128 = 1

_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int
_f32 = ctypes.c_float


class V6PlanC(ctypes.Structure):
    """Mirror of ``pgb_v6_plan``."""

    _fields_ = [
        ("sd", _vp),
        ("si", _vp),
        ("cta_ptr", _vp),
        ("n_cta", ctypes.c_int32),
        ("uniq", _vp),
        ("meta", _vp),
        ("w", _vp),
        ("sub_cap", ctypes.c_int32),
        ("gz", ctypes.c_int32),
        ("gy", ctypes.c_int32),
        ("gx", ctypes.c_int32),
        ("bz", ctypes.c_int32),
        ("by", ctypes.c_int32),
        ("bx", ctypes.c_int32),
        ("nbz", ctypes.c_int32),
        ("nby", ctypes.c_int32),
        ("nbx", ctypes.c_int32),
        ("zero_bricks", _vp),
        ("n_zero_bricks", ctypes.c_int32),
        ("cword", _vp),
        ("n_empty_tail", ctypes.c_int32),
    ]


class BrickPlanC(ctypes.Structure):
    """Mirror of ``pgb_brick_plan``."""

    _fields_ = [
        ("rep_src", _vp),
        ("rep_meta", _vp),
        ("rep_w", _vp),
        ("work", _vp),
        ("n_work", ctypes.c_int32),
        ("gz", ctypes.c_int32),
        ("gy", ctypes.c_int32),
        ("gx", ctypes.c_int32),
        ("bz", ctypes.c_int32),
        ("by", ctypes.c_int32),
        ("bx", ctypes.c_int32),
        ("nbz", ctypes.c_int32),
        ("nby", ctypes.c_int32),
        ("nbx", ctypes.c_int32),
        ("split_bricks", _vp),
        ("n_split_bricks", ctypes.c_int32),
    ]


# name -> argtypes (restype is always c_int status)
_SIGS = {
    "pgb_grog_interpolate": [_vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i32, _vp],
    "pgb_scatter_add": [_vp, _i64, _vp, _vp, _vp, _i64, _i32, _vp],
    "pgb_scatter_add_binned": [_vp, _i64, _vp, _vp, _vp, _i64, _vp, _i64, _i64, _i32, _vp],
    "pgb_gather": [_vp, _i64, _vp, _vp, _vp, _i64, _i32, _vp],
    "pgb_psf_scatter_scalar": [_vp, _i64, _vp, _vp, _i64, _i32, _vp],
    "pgb_psf_scatter_outer": [_vp, _i64, _i64, _vp, _vp, _vp, _i64, _i32, _vp],
    "pgb_psf_scatter_outer_basis": [_vp, _i64, _i64, _vp, _vp, _vp, _i64, _vp, _i64, _i32, _vp],
    "pgb_plan_geometry": [_vp, _i64, _i32, _vp, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "pgb_plan_gauss_sum": [_vp, _vp, _i64, _vp, _i64, _vp],
    "pgb_plan_weights": [_vp, _vp, _vp, _i64, _vp, _vp],
    "pgb_plan_quantize": [_vp, _i64, _i32, _f32, _f32, _f32, _i32, _i64, _vp, _vp],
    "pgb_grog_grid": [_vp, _i64, _vp, _i64, _vp, _i64, _i64, _i64, ctypes.POINTER(BrickPlanC), _vp],
    "pgb_grog_degrid": [
        _vp, _i64, _vp, _i64, _vp, _i64, _i64, _i64, ctypes.POINTER(BrickPlanC), _i32, _vp, _i64, _vp,
    ],
    "pgb_grog_expand": [_vp, _i64, _i32, _vp, _vp, _i64, _i64, _i64, _vp, _vp],
    "pgb_fft_expand": [_vp, _vp, _vp, _i64, _i64, _i32, _vp, _vp, _f32, _i32, _vp],
    "pgb_fft_combine": [_vp, _vp, _vp, _i64, _i64, _i32, _vp, _vp, _f32, _vp, _f32, _vp],
    "pgb_sparse_scatter": [_vp, _vp, _vp, _vp, _i64, _i64, _i64, _vp],
    "pgb_sparse_gather": [_vp, _vp, _vp, _vp, _i64, _i64, _i64, _vp],
    "pgb_psf_apply": [_vp, _vp, _i64, _i64, _vp],
    "pgb_fft_shift": [_vp, _vp, _vp, _i64, _i32, _vp, _f32, _i32, _vp],
    "pgb_dot_f64": [_vp, _vp, _i64, _vp, _vp, _i32, _i32, _vp],
    "pgb_cg_update_xr": [_vp, _vp, _vp, _vp, _i64, _vp, _vp],
    "pgb_cg_update_xr_rr": [_vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp],
    "pgb_cg_update_p": [_vp, _vp, _i64, _vp, _vp, _vp],
    "pgb_axpy": [_vp, _vp, _f32, _i64, _vp],
    "pgb_grog_grid_v8": [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _i64, _i64, _vp, _vp],
    "pgb_grog_degrid_v8": [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _i64, _i64, _vp, _vp, _vp, _i64, _vp],
    "pgb_subspace_scatter": [_vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _i64, _vp],
    "pgb_subspace_gather": [_vp, _vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _i64, _vp],
    "pgb_psf_apply_kk": [_vp, _vp, _i64, _i64, _i64, _i64, _vp],
    "pgb_dot_f64_batched": [_vp, _vp, _i64, _i64, _vp, _vp, _i32, _i32, _vp],
    "pgb_cg_update_xr_batched": [_vp, _vp, _vp, _vp, _i64, _i64, _vp, _vp],
    "pgb_cg_update_xr_rr_batched": [_vp, _vp, _vp, _vp, _i64, _i64, _vp, _vp, _vp],
    "pgb_cg_update_p_batched": [_vp, _vp, _i64, _i64, _vp, _vp, _vp],
    "pgb_dot_f64_noalloc": [_vp, _vp, _i64, _i64, _vp, _vp],
    "pgb_grog_grid_v6": [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _i64, _i64, _vp, _vp],
    "pgb_grog_degrid_v6": [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _i64, _i64, _vp, _vp, _vp, _i64, _vp],
    "pgb_grog_grid_tc": [_vp, _i64, _vp, _i64, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _vp, _vp],
    "pgb_grog_degrid_tc": [_vp, _i64, _vp, _i64, _vp, _vp, _i64, _i64, _i64, _i64, _i64, _vp, _vp, _vp, _i64, _vp],
    "pgb_grog_tc_blocks_per_sm": [_i64, _i64],
    "pgb_grog_tc_use_tma": [_i64],
    "pgb_grog_tc_timeouts": [_vp, _i64],
    "pgb_grog_tc_wait_limit": [_i64, _vp],
    "pgb_shift_chain": [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _i64, _i64, _vp, _vp],
    "pgb_lsmr_u_update": [_vp, _vp, _i64, _vp, _vp, _vp],
    "pgb_lsmr_u_scale": [_vp, _i64, _vp, _vp],
    "pgb_lsmr_v_full": [_vp, _vp, _vp, _i64, _vp, _vp, _vp],
    "pgb_lsmr_scalars": [_vp, _vp],
    "pgb_lsmr_vec_update": [_vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp],
    "pgb_plan_pack_quarter_warps": [_vp, _vp, _vp, _i64, _i64, _vp, _vp],
    "pgb_plan_pack_rows": [_vp, _vp, _i64, _i64, _i64, _vp, _vp],
    "pgb_plan_lpt": [_vp, _i64, _i64, _vp],
    "pgb_coil_covariance": [_vp, _i64, _i64, _vp, _vp],
    "pgb_coil_cross_covariance": [_vp, _vp, _i64, _i64, _vp, _vp],
    "pgb_coil_compress": [_vp, _i64, _i64, _i64, _i64, _vp, _vp, _vp],
    "pgb_coil_compress_tc": [_vp, _i64, _i64, _i64, _i64, _vp, _vp, _vp],
}
_SIZE_FUNCS = {
    "pgb_grog_v6_smem_bytes": [_i64, _i64, _i64, _i64, _i64],
    "pgb_grog_v8_smem_bytes": [_i64, _i64, _i64, _i64, _i64],
    "pgb_grog_tc_smem_bytes": [_i64, _i64, _i64, _i64, _i64],
    "pgb_reduce_scratch_bytes": [],
    "pgb_lsmr_scratch_bytes": [],
}

_lib = None


def exported_names() -> list[str]:
    """Names of all entry points this binding expects the library to export."""
    return ["pgb_last_error", "pgb_version", *_SIGS.keys(), *_SIZE_FUNCS.keys()]


def load_library():
    """Load the shared library (no CUDA device needed to load it)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"pygrog_b200: CUDA library not built ({LIB_PATH}); run "
            "`python -m pygrog_b200.csrc.build` (there is no CPU fallback)"
        )
    lib = ctypes.CDLL(str(LIB_PATH), mode=os.RTLD_LOCAL | getattr(os, "RTLD_NOW", 2))
    lib.pgb_last_error.restype = ctypes.c_char_p
    lib.pgb_last_error.argtypes = []
    lib.pgb_version.restype = ctypes.c_char_p
    lib.pgb_version.argtypes = []
    for name, argt in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = argt
        fn.restype = ctypes.c_int
    for name, argt in _SIZE_FUNCS.items():
        fn = getattr(lib, name)
        fn.argtypes = argt
        fn.restype = ctypes.c_size_t
    _lib = lib
    return lib


def lib():
    return load_library()


def check(status: int, what: str = "") -> None:
    if status != 0:
        msg = load_library().pgb_last_error().decode(errors="replace")
        raise RuntimeError(f"{what or 'pygrog_b200'}: {msg or 'error code %d' % status}")


def call(name: str, *args) -> None:
    """Call ``name`` with ``args`` and raise RuntimeError on a non-zero status."""
    st = getattr(load_library(), name)(*args)
    check(st, name)


def tc_timeouts(reset: bool = True) -> int:
    """Tile waits of the tensor-core adjoint that gave up since the last reset
    (device counter; the read is synchronous)."""
    n = ctypes.c_int64(0)
    call("pgb_grog_tc_timeouts", ctypes.byref(n), 1 if reset else 0)
    return int(n.value)


def check_tc_timeouts(what: str) -> None:
    """Raise RuntimeError if a tensor-core tile wait gave up since the last
    check.  A CTA whose wait gives up returns without writing the rest of its
    results, so the output of the call that launched it is incomplete.  Reads
    and resets the counter; the caller synchronises the launching stream
    first."""
    n = tc_timeouts(reset=True)
    if n:
        raise RuntimeError(
            f"{what}: {n} tensor-core tile wait(s) timed out; the result is incomplete "
            "(the brick tiles' tensor copies did not complete within the spin limit)"
        )


def stream_ptr(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def require_cuda(*tensors: torch.Tensor, what: str = "pygrog_b200") -> None:
    for t in tensors:
        if t is not None and t.device.type != "cuda":
            raise RuntimeError(
                f"{what}: tensors must be on a CUDA device (pygrog_b200 has no CPU path); "
                f"got device {t.device}"
            )


def dtype_code(t: torch.Tensor, what: str) -> int:
    if t.dtype in (torch.complex64, torch.float32):
        return PGB_C64
    if t.dtype in (torch.complex128, torch.float64):
        return PGB_C128
    raise RuntimeError(f"{what}: expected ComplexFloat or ComplexDouble, got {t.dtype}")
