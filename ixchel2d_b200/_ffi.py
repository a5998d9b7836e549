"""ctypes binding of libixb.so (include/ixb.h).

The library is loaded from the package directory; a missing library is an
error (there is no CPU fallback for the hot path).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("IXB_LIB", _PKG / "libixb.so"))

from ._types import (  # noqa: F401,E402  (re-exported)
    BC_DIRI, BC_NEUM, BC_OTHER, BODY_BOX, BODY_CHIME, BODY_CUADR, BODY_REGION, BODY_TEMP, BODY_TRIAN, BODY_VEL,
    EBC, ECUDA, EINVAL, EIO, ENOMEM, ENONFINITE, ESTATE, ETIMEOUT, MESH_CENT, MESH_TANH, MESH_TUBO, MESH_UNIF,
    NOALLOC_MAX_ELEMS, OK, PREC_FP32_REFINED, PREC_FP64, SOLVER_EXACT, SOLVER_HYBRID, VAR_T, VAR_U, VAR_V,
    BCSide, NuMonitor, Params, Report,
)


class IxbError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        msg = lib.ixb_strerror(status).decode() if lib is not None else str(status)
        super().__init__(f"{what}: status {status} ({msg})")


_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_vp = C.c_void_p

# (name, restype, argtypes) of every symbol declared in include/ixb.h
SIGNATURES = [
    ("ixb_version", C.c_int, []),
    ("ixb_strerror", C.c_char_p, [C.c_int]),
    ("ixb_device_count", C.c_int, []),
    ("ixb_create", C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(_vp)]),
    ("ixb_destroy", C.c_int, [_vp]),
    ("ixb_set_stream", C.c_int, [_vp, _vp]),
    ("ixb_set_mesh", C.c_int, [_vp, _dp, _dp, _dp, _dp]),
    ("ixb_set_params", C.c_int, [_vp, C.POINTER(Params)]),
    ("ixb_set_bc", C.c_int, [_vp, C.c_int, C.POINTER(BCSide)]),
    ("ixb_set_sources", C.c_int, [_vp, C.c_int, _dp, _dp]),
    ("ixb_upload_state", C.c_int, [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    ("ixb_download_state", C.c_int, [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    ("ixb_download_state_async", C.c_int, [_vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    ("ixb_download_wait", C.c_int, [_vp]),
    ("ixb_host_alloc", C.c_int, [C.c_size_t, C.POINTER(_vp)]),
    ("ixb_host_free", C.c_int, [_vp]),
    ("ixb_download_aux", C.c_int, [_vp, _dp, _dp, _dp, _dp, _dp]),
    ("ixb_simple_iterations", C.c_int, [_vp, C.c_int, C.POINTER(Report)]),
    ("ixb_simple_loop", C.c_int, [_vp, C.POINTER(Report)]),
    ("ixb_simple_converge", C.c_int, [_vp, C.POINTER(NuMonitor), C.POINTER(Report), _dp, _dp]),
    ("ixb_roll", C.c_int, [_vp]),
    ("ixb_step", C.c_int, [_vp, C.POINTER(Report)]),
    ("ixb_phase", C.c_int, [_vp, C.c_int]),
    ("ixb_set_work", C.c_int, [_vp, _dp, _dp, _dp]),
    ("ixb_time_phases", C.c_int, [_vp, C.c_int, C.c_size_t, _dp]),
    ("ixb_set_sweep_shape", C.c_int, [_vp, C.c_int, C.c_int, C.c_int]),
    ("ixb_autotune", C.c_int, [_vp, C.c_int, C.c_size_t, C.POINTER(C.c_int), _dp]),
    ("ixb_nusselt_y", C.c_int, [_vp, C.c_int, C.c_int, _dp, _dp]),
    ("ixb_nusselt_x", C.c_int, [_vp, C.c_int, C.c_int, _dp, _dp]),
    ("ixb_tridiag_f64", C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
    ("ixb_tridiag_f32", C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
    ("ixb_tridiag_f64_noalloc", C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
    ("ixb_batch_create", C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int, C.POINTER(_vp)]),
    ("ixb_batch_destroy", C.c_int, [_vp]),
    ("ixb_batch_instance", C.c_int, [_vp, C.c_int, C.POINTER(_vp)]),
    ("ixb_batch_set_sweep_shape", C.c_int, [_vp, C.c_int, C.c_int, C.c_int]),
    ("ixb_batch_autotune", C.c_int, [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    ("ixb_batch_restart", C.c_int, [_vp]),
    ("ixb_batch_iterate", C.c_int, [_vp, C.c_int, C.POINTER(C.c_int)]),
    ("ixb_batch_report", C.c_int, [_vp, C.c_int, C.POINTER(Report)]),
    ("ixb_adjoint_simple", C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp]),
    ("ixb_energy_iterations", C.c_int, [_vp, C.c_int]),
    ("ixb_adjoint_energy", C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _vp]),
    ("ixb_adjoint_energy_coupled", C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp]),
    ("ixb_set_bc_values", C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    ("ixb_mesh_axis", C.c_int, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _vp]),
    ("ixb_staggered_mesh", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_double, C.c_double,
                                     C.c_double, _vp, _vp, _vp, _vp]),
    ("ixb_write_state_files", C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_int] + [_vp] * 8 +
     [C.c_int, C.c_int, C.c_int, C.c_double]),
    ("ixb_read_state_files", C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_int] + [_vp] * 8 +
     [C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    ("ixb_tridiag_status", C.c_int, []),
    ("ixb_tridiag_set_first_wait_limit", C.c_int, [C.c_int]),
    ("ixb_iteration_launches", C.c_int, [_vp, C.POINTER(C.c_int)]),
    ("ixb_body_sources", C.c_int, [C.c_int, C.c_int, _vp, _vp, C.c_int, _vp, C.c_int, C.c_double] + [_vp] * 6),
    ("ixb_bc_locate", C.c_int, [C.c_int, C.c_int, _dp, C.POINTER(C.c_int), _dp, _dp, C.c_int, _dp, C.c_int,
                                C.POINTER(BCSide)]),
    ("ixb_read_bc_file", C.c_int, [C.c_char_p, _dp, C.c_int, _dp, C.c_int, C.POINTER(BCSide)]),
]


def _load():
    if not LIB_PATH.exists():
        raise ImportError(f"libixb.so not found at {LIB_PATH}; build it with `python -m ixchel2d_b200.build`")
    h = C.CDLL(str(LIB_PATH))
    for name, res, args in SIGNATURES:
        f = getattr(h, name)
        f.restype = res
        f.argtypes = args
    return h


lib = _load()


def check(status: int, what: str) -> None:
    if status != OK:
        raise IxbError(status, what)


def dptr(a: np.ndarray | None):
    """double* of a contiguous float64 array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.flags.c_contiguous)
    return a.ctypes.data_as(_dp)
