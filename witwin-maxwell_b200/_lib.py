"""ctypes binding of ``libfdtd_b200.so`` (the C ABI in ``include/fdtd_b200.h``).

The library is the only compute path of this package: if it is missing or
fails to load, every entry point raises instead of falling back to any CPU
implementation.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfdtd_b200.so"

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_i64_p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double
_i64 = ctypes.c_int64


class FdtdGridDesc(ctypes.Structure):
    _fields_ = [
        ("nx", _i),
        ("ny", _i),
        ("nz", _i),
        ("dt", _d),
        ("boundary", _i * 6),
        ("pml_lo", _i * 3),
        ("pml_hi", _i * 3),
        ("sample_block", _i),
        ("tile_rows", _i),
        ("chunk_planes", _i),
    ]


_SIGNATURES = {
    "fdtd_last_error": ([], ctypes.c_char_p),
    "fdtd_version": ([], ctypes.c_char_p),
    "fdtd_engine_create": ([ctypes.POINTER(FdtdGridDesc), _vp, ctypes.POINTER(_vp)], _i),
    "fdtd_engine_destroy": ([_vp], _i),
    "fdtd_bloch_create": ([_vp, _vp, ctypes.POINTER(_f), ctypes.POINTER(_f), ctypes.POINTER(_vp)], _i),
    "fdtd_bloch_destroy": ([_vp], _i),
    "fdtd_bloch_step_range": ([_vp, _i, _i], _i),
    "fdtd_bloch_last_ms": ([_vp, ctypes.POINTER(_f)], _i),
    "fdtd_batch_create": ([_vp, _i, _vp, ctypes.POINTER(_vp)], _i),
    "fdtd_batch_destroy": ([_vp], _i),
    "fdtd_batch_autotune": ([_vp], _i),
    "fdtd_batch_step_range": ([_vp, _i, _i], _i),
    "fdtd_batch_last_ms": ([_vp, ctypes.POINTER(_f)], _i),
    "fdtd_batch_info": ([_vp, _c_int_p, _c_int_p, _c_i64_p], _i),
    "fdtd_engine_set_storage": ([_vp, _i, _vp], _i),
    "fdtd_engine_get_storage": ([_vp, _c_int_p, _vp], _i),
    "fdtd_engine_set_spacing": ([_vp, _i, _vp, _vp], _i),
    "fdtd_engine_set_cpml": ([_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp], _i),
    "fdtd_engine_set_coefficients": ([_vp, _i, _vp, _f, _vp, _f], _i),
    "fdtd_engine_pack_field": ([_vp, _i, _vp], _i),
    "fdtd_engine_unpack_field": ([_vp, _i, _vp], _i),
    "fdtd_engine_pack_psi": ([_vp, _i, _i, _vp], _i),
    "fdtd_engine_unpack_psi": ([_vp, _i, _i, _vp], _i),
    "fdtd_engine_add_pole": ([_vp, _i, _i, _c_int_p, _vp, _vp, _f, _f, _c_int_p], _i),
    "fdtd_engine_pole_state": ([_vp, _i, _vp, _vp], _i),
    "fdtd_engine_set_pole_state": ([_vp, _i, _vp, _vp], _i),
    "fdtd_engine_add_patch": ([_vp, _i, _c_int_p, _vp, _vp, _i, _f], _i),
    "fdtd_engine_add_shifted_patch": ([_vp, _i, _c_int_p, _vp, _vp, _d, _i, _d, _d, _d, _d, _d, _i], _i),
    "fdtd_engine_set_nonlinear": ([_vp, _i, _i, _vp, _vp, _i, _f], _i),
    "fdtd_engine_set_full_aniso": ([_vp, _i, _c_int_p, _vp, _vp], _i),
    "fdtd_engine_add_aux_line": ([_vp, _i, _vp, _vp, _vp, _vp, _i, _vp, _i, _c_int_p], _i),
    "fdtd_engine_add_line_patch": ([_vp, _i, _c_int_p, _vp, _i, _i, _vp, _i, _f], _i),
    "fdtd_engine_add_sample_region": ([_vp, _i, _c_int_p, _c_i64_p], _i),
    "fdtd_engine_set_dft": ([_vp, _i, ctypes.POINTER(_d), _i, ctypes.POINTER(_d)], _i),
    "fdtd_engine_set_dft_windows": ([_vp, _i, ctypes.POINTER(_d), _i, ctypes.POINTER(_d)], _i),
    "fdtd_engine_read_dft": ([_vp, _vp, _vp], _i),
    "fdtd_engine_finalize": ([_vp], _i),
    "fdtd_engine_step_range": ([_vp, _i, _i], _i),
    "fdtd_engine_flush": ([_vp], _i),
    "fdtd_engine_checkpoint_save": ([_vp, _i], _i),
    "fdtd_engine_checkpoint_load": ([_vp, _i], _i),
    "fdtd_engine_autotune": ([_vp, _c_int_p, _c_int_p], _i),
    "fdtd_engine_info": ([_vp, _c_int_p, _c_int_p, _c_int_p, _c_int_p, _c_int_p, _c_i64_p], _i),
    "fdtd_engine_last_ms": ([_vp, ctypes.POINTER(_f)], _i),
    "fdtd_engine_time_kernel": ([_vp, _i, _i, ctypes.POINTER(_f)], _i),
    "fdtd_engine_set_launch": ([_vp, _i, _i, _i], _i),
    "fdtd_engine_get_launch": ([_vp, _c_int_p, _c_int_p, _c_int_p], _i),
    "fdtd_engine_set_prefetch": ([_vp, _i], _i),
    "fdtd_engine_set_wait_limit": ([_vp, _i], _i),
    "fdtd_engine_set_ade_pass": ([_vp, _i], _i),
    "fdtd_engine_checkpoint_reserve": ([_vp, _i], _i),
    "fdtd_engine_adjoint_init": ([_vp, _c_int_p, _i], _i),
    "fdtd_engine_adjoint_set_seed": ([_vp, _vp, _vp], _i),
    "fdtd_engine_replay_range": ([_vp, _i, _i], _i),
    "fdtd_engine_step_range_recorded": ([_vp, _i, _i], _i),
    "fdtd_engine_adjoint_range": ([_vp, _i, _i], _i),
    "fdtd_engine_backward_replay": ([_vp, _i, _i], _i),
    "fdtd_engine_set_replay_region": ([_vp, _i], _i),
    "fdtd_engine_set_range_flush": ([_vp, _i], _i),
    "fdtd_engine_get_plane": ([_vp, _i, _i, _vp], _i),
    "fdtd_engine_set_plane": ([_vp, _i, _i, _vp], _i),
    "fdtd_engine_adjoint_grad": ([_vp, _i, _vp], _i),
    "fdtd_engine_adjoint_pack": ([_vp, _i, _i, _i, _vp], _i),
    "fdtd_engine_adjoint_unpack": ([_vp, _i, _i, _i, _vp], _i),
    "fdtd_op_update_magnetic": (
        [_i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _f, _f, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_int_p, _vp],
        _i,
    ),
    "fdtd_op_update_electric": (
        [_i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _f, _f, _vp, _vp, _c_int_p, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_int_p, _vp],
        _i,
    ),
    "fdtd_op_update_debye": ([_i64, _vp, _vp, _f, _f, _vp, _vp, _vp], _i),
    "fdtd_op_update_drude": ([_i64, _vp, _vp, _f, _vp, _vp], _i),
    "fdtd_op_update_lorentz": ([_i64, _vp, _vp, _f, _f, _f, _vp, _vp, _vp], _i),
    "fdtd_op_apply_polarization": ([_i64, _vp, _vp, _f, _vp, _vp], _i),
    "fdtd_op_update_electric_full_aniso": ([_i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i,
                                            _vp], _i),
    "fdtd_op_update_kerr_curl": ([_i, _c_int_p, _vp, _vp, _vp, _vp, _vp, _vp, _f, _f, _vp, _vp], _i),
    "fdtd_op_update_nonlinear_coefficients": ([_i, _c_int_p, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _f, _f,
                                               _vp, _vp, _vp], _i),
    "fdtd_op_add_source_patch": ([_vp, _c_int_p, _vp, _c_int_p, _c_int_p, _f, _vp], _i),
    "fdtd_op_update_electric_bloch": ([_i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _f, _f, _f, _f,
                                      _vp, _vp, _i, _i, _vp], _i),
    "fdtd_op_apply_cpml_z_correction": ([_i, _vp, _c_int_p, _vp, _c_int_p, _vp, _vp, _vp, _vp, _vp, _vp, _c_int_p,
                                         _i, _i, _i, _i, _vp], _i),
    "fdtd_op_project_periodic": ([_vp, _c_int_p, _i, _vp], _i),
    "fdtd_op_project_bloch": ([_vp, _vp, _c_int_p, _i, _f, _f, _vp], _i),
    "fdtd_pp_diffraction": ([_i, _i, _vp, _vp, _vp, _i, _vp, _i, _vp, _vp, _vp, _vp], _i),
    "fdtd_pp_nfft": ([_i, _vp, _vp, _vp, _i, _vp, _vp, _d, _d, _vp, _vp, _vp, _vp], _i),
    "fdtd_op_add_cw_patch": ([_vp, _c_int_p, _vp, _vp, _c_int_p, _c_int_p, _f, _f, _vp], _i),
    "fdtd_op_add_shifted_patch": ([_vp, _c_int_p, _vp, _vp, _vp, _i, _c_int_p, _c_int_p, _i, _f, _f, _f, _f, _f, _f,
                                   _vp], _i),
    "fdtd_op_add_line_patch": ([_vp, _c_int_p, _vp, _c_int_p, _c_int_p, _vp, _vp, _i, _f, _vp], _i),
    "fdtd_op_aux_magnetic": ([_i, _vp, _vp, _vp, _vp, _vp], _i),
    "fdtd_op_aux_electric": ([_i, _vp, _vp, _vp, _vp, _i, _f, _vp], _i),
    "fdtd_op_aux_line_history_static": ([_i, _vp, _vp, _vp, _vp, _i, _vp, _i, _vp, _vp, _vp], _i),
    "fdtd_op_point_observers": ([_vp, _c_int_p, _i, _vp, _vp, _vp, _vp, _vp, _f, _f, _vp], _i),
    "fdtd_op_plane_observer": ([_vp, _c_int_p, _i, _i, _vp, _vp, _f, _f, _vp], _i),
    "fdtd_op_dft_volume": ([_i64, _i, _vp, _vp, _vp, _vp, _vp, _vp], _i),
    "fdtd_op_clamp_face": ([_vp, _c_int_p, _i, _i, _vp], _i),
}

EXPORTED_SYMBOLS = tuple(_SIGNATURES)

_lib = None
_lock = threading.Lock()


class FdtdError(RuntimeError):
    """A non-zero status returned by the C ABI."""


def load(path: Path | str | None = None) -> ctypes.CDLL:
    """Load the shared library (once) and declare every exported signature."""
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        lib_path = Path(path) if path is not None else LIB_PATH
        if not lib_path.exists():
            raise FdtdError(
                f"{lib_path} is missing: build it with `python witwin-maxwell_b200/build.py` "
                "(there is no CPU fallback)"
            )
        lib = ctypes.CDLL(str(lib_path))
        for name, (argtypes, restype) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = restype
        if path is None:
            _lib = lib
        return lib


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        lib = load()
        msg = lib.fdtd_last_error().decode(errors="replace")
        raise FdtdError(f"{what or 'fdtd call'} failed with status {rc}: {msg}")


def int_array(values) -> ctypes.Array:
    values = [int(v) for v in values]
    return (ctypes.c_int * len(values))(*values)


def ptr(tensor) -> int | None:
    """Device pointer of a torch tensor (None for None)."""
    if tensor is None:
        return None
    return int(tensor.data_ptr())
