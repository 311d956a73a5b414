"""ctypes binding of ``liboem_b200.so`` (declarations in ``include/oem_b200.h``).

The library is loaded from the package directory. There is no fallback: if it is missing or
does not load, every entry point raises, so a run can never silently fall back to CPU code.
Status codes map to exceptions the way OpenEM's solver fails closed: unsupported physics ->
``NotImplementedError``, bad input -> ``ValueError``, device trouble -> ``RuntimeError``.
"""

from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

LIB_PATH = pathlib.Path(__file__).resolve().parent / "liboem_b200.so"

OK, ERR_INVALID, ERR_UNSUPPORTED, ERR_CUDA, ERR_TIMEOUT, ERR_STATE, ERR_NOMEM = 0, -1, -2, -3, -4, -5, -6

#: Every symbol the header declares, with (restype, argtypes).
_P = C.c_void_p
_I = C.c_int
_L = C.c_int64
_D = C.c_double
SIGNATURES = {
    "oem_version": (_I, []),
    "oem_last_error": (C.c_char_p, []),
    "oem_plan_create": (_I, [_I, _I, _I, _I, _D, _D, C.POINTER(_P)]),
    "oem_plan_destroy": (_I, [_P]),
    "oem_plan_set_axis": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I]),
    "oem_plan_set_materials": (_I, [_P, _I, _P, _I, _P]),
    "oem_plan_set_materials_device": (_I, [_P, _I, _P, _I, _P]),
    "oem_plan_set_pole_sets": (_I, [_P, _I, _P, _P, _P, _L, _L]),
    "oem_plan_set_pole_sets_device": (_I, [_P, _I, _P, _P, _P, _L, _L]),
    "oem_plan_add_plane_source": (_I, [_P, _I, _I, _I, _D, _D, _L, _P, _P]),
    "oem_plan_add_dipoles": (_I, [_P, _I, _I, _P, _P, _P, _P, _I, _L, _P]),
    "oem_plan_add_dipoles_complex": (_I, [_P, _I, _I, _P, _P, _P, _P, _I, _L, _P, _P]),
    "oem_plan_add_mode_source": (_I, [_P, _I, _I, _I, _I, _I, _D, _D, _D, _D, _I, _P, _L,
                                      _P, _P]),
    "oem_plan_set_axis_phase": (_I, [_P, _I, _P, _P]),
    "oem_plan_add_absorber": (_I, [_P, _I, _I, _I, _P, _P]),
    "oem_plan_set_xchunk": (_I, [_P, _I]),
    "oem_plan_set_wait_expiry_check": (_I, [_P, _I]),
    "oem_plan_enable_checkpoints": (_I, [_P, _I]),
    "oem_plan_set_gradient_box": (_I, [_P, _P]),
    "oem_plan_add_tensor": (_I, [_P, _I, _P, _P, _P, _P, _P]),
    "oem_plan_add_dispersion_mix": (_I, [_P, _I, _P, _P, _P, _P, _I, _P, _P, _I, _P, _D]),
    "oem_plan_add_tfsf": (_I, [_P, _I, _P, _I, _P, _I, _I, _P, _I, _I, _P]),
    "oem_plan_add_flux_time_monitor": (_I, [_P, _I, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P,
                                            _I, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _P]),
    "oem_plan_read_flux_time": (_I, [_P, _I, _P, _P]),
    "oem_plan_add_modulation": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P, _D]),
    "oem_plan_adjoint_flux": (_I, [_P, _I, _P, _P, _P, _P, _P, _P]),
    "oem_plan_adjoint_flux_box": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _P]),
    "oem_plan_add_flux_monitor": (_I, [_P, _I, _I, _I, _L, _P, _I, C.POINTER(_I)]),
    "oem_plan_add_box_monitor": (_I, [_P, _I, _I, _I, _I, _I, _I, _I, _L, _P, _I,
                                      C.POINTER(_I)]),
    "oem_plan_add_time_monitor": (_I, [_P, _I, _P, _I, _I, _I, _I, _I, _I, _I, _I, _I, _I,
                                       C.POINTER(_I)]),
    "oem_plan_finalize": (_I, [_P, _L]),
    "oem_plan_run": (_I, [_P, _L, _P]),
    "oem_plan_flush": (_I, [_P, _P]),
    "oem_plan_status": (_I, [_P, _P]),
    "oem_plan_launches_per_step": (_I, [_P, C.POINTER(_I)]),
    "oem_plan_box_snapshots_in_update": (_I, [_P, C.POINTER(_I)]),
    "oem_plan_pole_pass_ahead": (_I, [_P, C.POINTER(_I)]),
    "oem_plan_steps": (_I, [_P, C.POINTER(_L)]),
    "oem_plan_read_monitor": (_I, [_P, _I, _P, _P, _P]),
    "oem_plan_read_monitor_interleaved": (_I, [_P, _I, _P, _P]),
    "oem_plan_readout_nonfinite": (_I, [_P, C.POINTER(_L)]),
    "oem_plan_read_time_monitor": (_I, [_P, _I, _P, _P]),
    "oem_plan_read_field": (_I, [_P, _I, _P, _P]),
    "oem_plan_read_field_complex": (_I, [_P, _I, _P, _P, _P]),
    "oem_plan_read_time_monitor_complex": (_I, [_P, _I, _P, _P, _P]),
    "oem_plan_write_field": (_I, [_P, _I, _P, _P]),
    "oem_plan_write_field_complex": (_I, [_P, _I, _P, _P, _P]),
    "oem_plan_energy": (_I, [_P, _P, _P]),
    "oem_plan_field_ptrs": (_I, [_P, _P, C.POINTER(_I)]),
    "oem_field_energy_noalloc": (_I, [_P, _P, _I, _I, _I, _I, _P, _P, _P]),
    "oem_plan_enable_timing": (_I, [_P, _I]),
    "oem_plan_timing": (_I, [_P, _I, _P, _P, _P, C.POINTER(_I)]),
}

_lib = None


def load():
    """Load the library once and declare every entry point. Raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH.name} is not built; run `python -m openem_b200.build`")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().oem_last_error().decode(errors="replace")


def check(rc: int, what: str = "") -> None:
    if rc == OK:
        return
    msg = f"{what}: {last_error()}" if what else last_error()
    if rc == ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if rc in (ERR_INVALID,):
        raise ValueError(msg)
    raise RuntimeError(f"[oem status {rc}] {msg}")


def ptr(a: np.ndarray | None):
    """Host pointer of a C-contiguous array (kept alive by the caller)."""
    if a is None:
        return None
    assert a.flags.c_contiguous, "array must be C-contiguous"
    return C.c_void_p(a.ctypes.data)


def stream_handle(stream) -> C.c_void_p:
    """``cudaStream_t`` of a torch stream, an int handle, or None (legacy default stream)."""
    if stream is None:
        return C.c_void_p(0)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(int(stream.cuda_stream))
