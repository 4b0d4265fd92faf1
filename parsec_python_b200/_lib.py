"""ctypes binding of libpsc.so (the C ABI declared in include/psc.h).

The library is built in-tree (``parsec_python_b200/libpsc.so``) by
``parsec_python_b200.build``.  There is no fallback: if the library is
missing or does not load, every GPU entry point raises.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int, c_long, c_ulonglong, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpsc.so"

F64 = 0
F32 = 1

_P = c_void_p
_SIGS = {
    "psc_version": ([], c_int),
    "psc_launch_count": ([], ctypes.c_longlong),
    "psc_last_error": ([_P], ctypes.c_char_p),
    "psc_ctx_create": ([c_int, c_int, c_int, c_double, c_int, POINTER(_P)], c_int),
    "psc_ctx_destroy": ([_P], c_int),
    "psc_ctx_info": ([_P, POINTER(c_long)], c_int),
    "psc_status": ([_P, POINTER(c_int), c_int, _P], c_int),
    "psc_set_species": ([_P, c_int, c_int, _P, c_double, c_double], c_int),
    "psc_spline_coeffs": ([c_int, _P, _P, POINTER(c_int), _P, _P, _P, _P], c_int),
    "psc_sad_setup": ([_P, c_int, _P, _P, c_double, c_double, c_double, c_double, _P, _P, _P, _P, _P], c_int),
    "psc_projector_setup": ([_P, c_int, _P, _P, c_double, _P], c_int),
    "psc_ml_density": ([_P, _P, c_double, c_double, c_double, _P, c_double, _P, _P, _P, _P], c_int),
    "psc_projector_export": ([_P, _P, _P, _P, _P], c_int),
    "psc_numpy_sum": ([_P, _P, c_long, _P, _P], c_int),
    "psc_set_potential": ([_P, _P, _P], c_int),
    "psc_apply_h": ([_P, c_int, _P, c_long, _P, c_long, c_int, _P], c_int),
    "psc_apply_h_axpby": ([_P, c_int, _P, c_long, _P, c_long, _P, c_long, c_int, c_double, c_double, c_double, _P],
                          c_int),
    "psc_set_stencil_impl": ([_P, c_int], c_int),
    "psc_set_stencil_weights": ([_P, c_int], c_int),
    "psc_laplacian_apply": ([_P, _P, _P, c_int, c_long, _P], c_int),
    "psc_cheb_filter": ([_P, c_int, c_int, c_int, _P, _P, _P, c_long, c_int, POINTER(c_int), _P], c_int),
    "psc_lanczos_bound": ([_P, c_int, c_ulonglong, _P, _P], c_int),
    "psc_lanczos_bound_v": ([_P, c_int, _P, _P, _P], c_int),
    "psc_apply_nonlocal": ([_P, c_int, _P, c_long, _P, c_long, c_int, _P], c_int),
    "psc_lanczos_run": ([_P, _P, c_ulonglong, c_int, c_int, _P, c_long, _P, _P], c_int),
    "psc_tridiag_eig": ([_P, _P, c_int, c_int, _P, _P, c_long, _P], c_int),
    "psc_orthonormalize_rank": ([_P, c_int, _P, _P, c_long, c_int, c_double, POINTER(c_int), POINTER(c_int), _P],
                                c_int),
    "psc_filter_bounds": ([_P, c_int, _P, c_int, _P, _P, _P], c_int),
    "psc_orthonormalize": ([_P, c_int, _P, _P, c_long, c_int, c_int, POINTER(c_int), _P], c_int),
    "psc_rayleigh_ritz": ([_P, c_int, _P, _P, c_long, c_int, _P, _P], c_int),
    "psc_subspace_rr": ([_P, c_int, _P, _P, c_long, c_int, _P, _P], c_int),
    "psc_gram": ([_P, c_int, _P, c_long, _P, c_long, c_int, c_int, _P, _P], c_int),
    "psc_gemm_nn": ([_P, c_int, _P, c_long, c_int, _P, c_int, _P, c_long, _P], c_int),
    "psc_syev": ([_P, _P, c_int, _P, _P, _P], c_int),
    "psc_occupations": ([_P, _P, c_int, c_double, c_double, c_double, _P, _P, _P], c_int),
    "psc_density": ([_P, c_int, _P, c_long, c_int, _P, _P, c_double, c_double, _P, _P, _P], c_int),
    "psc_pcg_poisson": ([_P, _P, _P, c_int, c_double, POINTER(c_int), _P], c_int),
    "psc_set_use_graphs": ([_P, c_int], c_int),
    "psc_pcg_poisson_prec": ([_P, _P, _P, c_int, c_double, POINTER(c_int), _P], c_int),
    "psc_poisson_precond": ([_P, _P, _P, _P], c_int),
    "psc_lda_xc": ([_P, _P, _P, c_double, _P, _P], c_int),
    "psc_lda_xc_noalloc": ([_P, _P, c_long, c_double, _P, _P], c_int),
    "psc_set_gram_impl": ([_P, c_int], c_int),
    "psc_set_gram_chunk": ([_P, c_long], c_int),
    "psc_set_gemm_impl": ([_P, c_int], c_int),
    "psc_set_wait_limit": ([_P, c_long], c_int),
    "psc_set_sphere_mask": ([_P, c_double, _P], c_int),
    "psc_mask_block": ([_P, c_int, _P, c_long, c_int, _P], c_int),
    "psc_gram_pair": ([_P, c_int, _P, _P, c_long, c_int, _P, _P, _P], c_int),
    "psc_conv3d_fwd": ([_P, _P, _P, _P, _P, _P, c_int, _P, _P, _P], c_int),
    "psc_set_conv_impl": ([_P, c_int], c_int),
    "psc_conv3d_bwd": ([_P, _P, _P, _P, _P, _P, _P, c_int, _P, _P, _P, c_int, _P, c_int, _P, _P, _P, c_long, _P],
                       c_int),
    "psc_mse_loss": ([_P, _P, c_int, _P, c_long, _P, _P, _P], c_int),
    "psc_adam_step": ([_P, _P, _P, _P, _P, _P, c_long, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                       ctypes.c_float, c_int, _P], c_int),
    "psc_f32_to_bf16": ([_P, _P, _P, c_long, _P], c_int),
    "psc_pack_input": ([_P, _P, _P, c_double, c_double, _P, _P], c_int),
    "psc_scf_update": ([_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P], c_int),
    "psc_mixer_reset": ([_P, c_int], c_int),
    "psc_mixer_step": ([_P, _P, _P, c_double, c_double, _P, POINTER(c_int), _P], c_int),
    "psc_mixer_history": ([_P, POINTER(c_int)], c_int),
    "psc_mix2_diff": ([_P, _P, _P, _P, _P, c_double, _P], c_int),
    "psc_mix2_store": ([_P, _P, _P, _P, _P, _P], c_int),
    "psc_block_dots": ([_P, _P, c_long, c_int, _P, _P, _P], c_int),
    "psc_block_combine": ([_P, _P, _P, _P, c_double, _P, c_long, c_int, _P, _P], c_int),
    "psc_block_absrow_max": ([_P, _P, c_long, c_int, _P, _P], c_int),
    "psc_random": ([_P, c_int, c_int, c_ulonglong, _P, c_long, c_long, c_int, _P], c_int),
    "psc_cast": ([_P, c_int, _P, _P, c_long, _P], c_int),
    "psc_dot": ([_P, _P, _P, c_long, _P, _P], c_int),
    "psc_axpby": ([_P, _P, _P, c_double, c_double, _P, c_long, _P], c_int),
}

_lib = None


class PscError(RuntimeError):
    """An error status returned by libpsc."""


def load() -> ctypes.CDLL:
    """Load libpsc.so once; raise if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise PscError(f"{LIB_PATH} is missing: build it with `python -m parsec_python_b200.build` "
                       "(the GPU path has no fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def check(rc: int, ctx=None, what: str = "") -> None:
    if rc != 0:
        msg = load().psc_last_error(ctx)
        text = msg.decode() if msg else "unknown error"
        raise PscError(f"{what or 'libpsc'} failed (status {rc}): {text}")


def call(name: str, *args, ctx=None) -> None:
    """Call a libpsc entry point that returns a status code and raise on error."""
    fn = getattr(load(), name)
    check(fn(*args), ctx, name)
