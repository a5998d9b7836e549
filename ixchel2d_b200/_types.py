"""Constants and ctypes structures of include/ixb.h.

This module loads no library: the synthetic-case builders and the CPU
oracle's callers use these types without mapping libixb.so.
"""
from __future__ import annotations

import ctypes as C

OK, EINVAL, ECUDA, ENONFINITE, ETIMEOUT, EBC, ESTATE, EIO, ENOMEM = range(9)
NOALLOC_MAX_ELEMS = 1 << 20
PREC_FP64, PREC_FP32_REFINED = 0, 1
SOLVER_HYBRID, SOLVER_EXACT = 0, 1
VAR_U, VAR_V, VAR_T = 0, 1, 2
BC_OTHER, BC_DIRI, BC_NEUM = 0, 1, 2
MESH_UNIF, MESH_TUBO, MESH_CENT, MESH_TANH = 0, 1, 2, 3
BODY_BOX, BODY_REGION, BODY_TRIAN, BODY_CUADR, BODY_CHIME = 0, 1, 2, 3, 4
BODY_VEL, BODY_TEMP = 1, 2


class Params(C.Structure):
    _fields_ = [
        ("gamma_momen", C.c_double), ("gamma_energ", C.c_double), ("Ri", C.c_double), ("Riy", C.c_double),
        ("dt", C.c_double), ("rel_vel", C.c_double), ("rel_pres", C.c_double), ("rel_ener", C.c_double),
        ("conv_u", C.c_double), ("conv_p", C.c_double), ("conv_t", C.c_double), ("conv_resi", C.c_double),
        ("conv_paso", C.c_double), ("p_update", C.c_double),
        ("iter_ecuaci_max", C.c_int), ("iter_simple_max", C.c_int), ("solver", C.c_int),
        ("reserved", C.c_int * 5),
    ]


class BCSide(C.Structure):
    _fields_ = [("side", C.c_int), ("ndivis", C.c_int), ("type", C.c_int * 15), ("value", C.c_double * 15),
                ("index", C.c_int * 16)]


class Report(C.Structure):
    _fields_ = [
        ("maxbo", C.c_double), ("residuo", C.c_double), ("err_u", C.c_double), ("err_p", C.c_double),
        ("err_t", C.c_double), ("n_simple", C.c_int64), ("n_momen", C.c_int64), ("n_pres", C.c_int64),
        ("n_ener", C.c_int64), ("exit_code", C.c_int), ("status", C.c_int),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class NuMonitor(C.Structure):
    _fields_ = [("vertical", C.c_int), ("k0", C.c_int), ("k1", C.c_int), ("wall", C.c_int), ("every", C.c_int),
                ("reserved", C.c_int), ("max_iters", C.c_int64), ("tol_dnu", C.c_double), ("tol_maxbo", C.c_double)]
