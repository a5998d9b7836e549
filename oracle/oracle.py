"""ctypes view of the CPU oracle (oracle/ixb_oracle.cpp).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
the CPU legs of bench.py, as the checker / CPU baseline.  Parity of the
oracle itself is unpinned against reference outputs (no Fortran compiler in
this image; the reference ships no golden vectors); known-answer tests in
tests/test_oracle.py pin it instead.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libixb_oracle.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def _load():
    if not LIB.exists():
        build()
    h = C.CDLL(str(LIB))
    sig = {
        "ixo_new": (_vp, [C.c_int, C.c_int]),
        "ixo_free": (None, [_vp]),
        "ixo_set_threads": (None, [C.c_int]),
        "ixo_max_threads": (C.c_int, []),
        "ixo_set_mesh": (C.c_int, [_vp, _dp, _dp, _dp, _dp]),
        "ixo_set_params": (C.c_int, [_vp, _dp, _ip]),
        "ixo_set_bc": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _ip, _dp, _ip]),
        "ixo_set_bc_values": (C.c_int, [_vp, C.c_int, C.c_int, _dp]),
        "ixo_set_sources": (C.c_int, [_vp, C.c_int, _dp, _dp]),
        "ixo_set_state": (C.c_int, [_vp] + [_dp] * 7),
        "ixo_get_state": (C.c_int, [_vp] + [_dp] * 7),
        "ixo_get_aux": (C.c_int, [_vp] + [_dp] * 5),
        "ixo_simple_iterations": (C.c_int, [_vp, C.c_int, _dp]),
        "ixo_simple_loop": (C.c_int, [_vp, _dp]),
        "ixo_roll": (C.c_int, [_vp]),
        "ixo_phase": (C.c_int, [_vp, C.c_int]),
        "ixo_set_corr_pres": (C.c_int, [_vp, _dp]),
        "ixo_set_auav": (C.c_int, [_vp, _dp, _dp]),
        "ixo_get_metric": (C.c_int, [_vp, C.c_int, _dp]),
        "ixo_tridiagonal": (None, [_dp, _dp, _dp, _dp, C.c_int]),
        "ixo_tridiagonal_batch": (None, [_dp, _dp, _dp, _dp, C.c_int, C.c_int]),
        "ixo_nusselt_y": (C.c_int, [_vp, _dp, C.c_int, C.c_int, _dp, _dp]),
        "ixo_nusselt_x": (C.c_int, [_vp, _dp, C.c_int, C.c_int, _dp, _dp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(h, name)
        f.restype = res
        f.argtypes = args
    return h


lib = _load()

PARAM_ORDER = ["gamma_momen", "gamma_energ", "Ri", "Riy", "dt", "rel_vel", "rel_pres", "rel_ener", "conv_u",
               "conv_p", "conv_t", "conv_resi", "conv_paso", "p_update"]
REPORT_KEYS = ["maxbo", "residuo", "err_u", "err_p", "err_t", "n_simple", "n_momen", "n_pres", "n_ener",
               "exit_code"]
STATE_KEYS = ("u", "v", "p", "T", "u_ant", "v_ant", "T_ant")
METRICS = ["deltaxp", "deltayp", "deltaxu", "deltayu", "deltaxv", "deltayv", "fexp", "feyp", "fexu", "feyv",
           "xu", "yv", "xp", "yp"]


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def set_threads(n: int) -> None:
    lib.ixo_set_threads(n)


def max_threads() -> int:
    return lib.ixo_max_threads()


def tridiagonal(a, b, c, r):
    """tridiagonal(a,b,c,r,n) in place on float64 copies; returns x."""
    a, b, c, r = (np.array(x, dtype=np.float64) for x in (a, b, c, r))
    lib.ixo_tridiagonal(_p(a), _p(b), _p(c), _p(r), a.size)
    return r


def definir_cuerpo(opcion: str, mi: int, nj: int, xp, yp) -> dict:
    """Penalty sources of an immersed body, restating definir_cuerpo
    (source/mod_front_inmersa.f90:54-179) loop by loop: for every p node
    (xp(ii), yp(jj)) inside the body, fuente_lin = -10.0e50 and fuente_con =
    10.0e50*10.0e-12 on u and v (T: 10e50*1.0 for 'chime') at (ii, jj).  The
    reference's writes to u at ii = mi+1 and v at jj = nj+1 fall outside
    those arrays and are dropped.  Returns var -> (fcon, flin), var 0/1/2 =
    u/v/T, in the Fortran shapes."""
    xp = [float(x) for x in xp]
    yp = [float(y) for y in yp]
    fu = np.zeros((mi, nj + 1), order="F"); lu = np.zeros_like(fu)
    fv = np.zeros((mi + 1, nj), order="F"); lv = np.zeros_like(fv)
    ft = np.zeros((mi + 1, nj + 1), order="F"); lt = np.zeros_like(ft)

    def recta_mxb1(x):  # :210-215
        mm = 1.0 / 2.0
        bb = -(0.1 - mm * 6.0) / mm
        return x / mm + bb

    def recta_mxb2(x):  # :226-231
        mm = -1.0 / 2.0
        bb = -(0.1 - mm * 6.0) / mm
        return x / mm + bb

    def en_region_tipo1(xx, yy, aa, bb, f1, f2):  # :188-207
        return aa <= xx <= bb and f1(xx) <= yy <= f2(xx)

    def put(ii, jj, temp):  # 1-based (ii, jj)
        if ii <= mi:
            lu[ii - 1, jj - 1] = -10.0e50
            fu[ii - 1, jj - 1] = 10.0e50 * 10.0e-12
        if jj <= nj:
            lv[ii - 1, jj - 1] = -10.0e50
            fv[ii - 1, jj - 1] = 10.0e50 * 10.0e-12
        if temp:
            lt[ii - 1, jj - 1] = -10e50
            ft[ii - 1, jj - 1] = 10e50 * 1.0

    if opcion == "trian":
        yv, hh = 0.1, 0.1
        for jj in range(1, nj + 2):
            if yv - hh <= yp[jj - 1] <= yv:
                for ii in range(1, mi + 2):
                    if en_region_tipo1(yp[jj - 1], xp[ii - 1], yv - hh, yv, recta_mxb1, recta_mxb2):
                        put(ii, jj, False)
    elif opcion in ("cuadr", "chime"):
        yv, xv, hh = (0.05, 6.0, 0.1) if opcion == "cuadr" else (0.5, 8.5, 0.3)
        for jj in range(1, nj + 2):
            if yv - hh / 2.0 <= yp[jj - 1] <= yv + hh / 2.0:
                for ii in range(1, mi + 2):
                    if xv - hh / 2.0 <= xp[ii - 1] <= xv + hh / 2.0:
                        put(ii, jj, opcion == "chime")
    return {0: (fu, lu), 1: (fv, lv), 2: (ft, lt)}


def tridiagonal_batch(a, b, c, d):
    """Independent contiguous systems (rows of 2-D arrays); returns x."""
    a, b, c, d = (np.array(x, dtype=np.float64, order="C") for x in (a, b, c, d))
    nsys, n = a.shape
    lib.ixo_tridiagonal_batch(_p(a), _p(b), _p(c), _p(d), n, nsys)
    return d


class OracleCase:
    """One case on the CPU oracle, mirroring ixchel2d_b200.Simple2D."""

    def __init__(self, case, **param_over):
        self.mi, self.nj = case.mi, case.nj
        self.h = lib.ixo_new(case.mi, case.nj)
        if not self.h:
            raise ValueError("grid too small")
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (case.xu, case.yv, case.xp, case.yp)]
        lib.ixo_set_mesh(self.h, *map(_p, arrs))
        prm = dict(case.params)
        prm.update(param_over)
        self.set_params(prm)
        for var, sides in case.bc.items():
            for b in sides:
                nd = b.ndivis
                ty = (C.c_int * 15)(*b.type)
                va = (C.c_double * 15)(*b.value)
                ix = (C.c_int * 16)(*b.index)
                lib.ixo_set_bc(self.h, var, b.side, nd, ty, va, ix)
        for var, (fc, fl) in case.sources.items():
            self.set_sources(var, fc, fl)
        self.set_state(case.state)

    def set_bc_values(self, var: int, side: int, values):
        """Per-line boundary values of one side (the extension of ixo_set_bc_values,
        mirroring the library's ixb_set_bc_values)."""
        a = np.ascontiguousarray(values, dtype=np.float64)
        if lib.ixo_set_bc_values(self.h, var, side, _p(a)) != 0:
            raise ValueError("ixo_set_bc_values")

    def energy_passes(self, n: int):
        """n passes of the two T sweeps (T-y, T-x) at the current u, v: the
        oracle side of the library's ixb_energy_iterations."""
        for _ in range(n):
            self.phase(7)
            self.phase(8)

    def set_params(self, prm: dict):
        d = (C.c_double * len(PARAM_ORDER))(*[float(prm[k]) for k in PARAM_ORDER])
        n = (C.c_int * 2)(int(prm["iter_ecuaci_max"]), int(prm["iter_simple_max"]))
        lib.ixo_set_params(self.h, d, n)

    def set_sources(self, var, fcon, flin):
        fc = None if fcon is None else np.asfortranarray(fcon, dtype=np.float64)
        fl = None if flin is None else np.asfortranarray(flin, dtype=np.float64)
        lib.ixo_set_sources(self.h, var, _p(fc), _p(fl))

    def set_state(self, st: dict):
        arrs = [None if st.get(k) is None else np.asfortranarray(st[k], dtype=np.float64) for k in STATE_KEYS]
        lib.ixo_set_state(self.h, *map(_p, arrs))

    def get_state(self) -> dict:
        mi, nj = self.mi, self.nj
        sh = {"u": (mi, nj + 1), "v": (mi + 1, nj), "p": (mi + 1, nj + 1), "T": (mi + 1, nj + 1),
              "u_ant": (mi, nj + 1), "v_ant": (mi + 1, nj), "T_ant": (mi + 1, nj + 1)}
        out = {k: np.zeros(s, order="F") for k, s in sh.items()}
        lib.ixo_get_state(self.h, *[_p(out[k]) for k in STATE_KEYS])
        return out

    def get_aux(self) -> dict:
        mi, nj = self.mi, self.nj
        out = {"au": np.zeros((mi, nj + 1), order="F"), "av": np.zeros((mi + 1, nj), order="F"),
               "b_o": np.zeros((mi + 1, nj + 1), order="F"), "Resu": np.zeros((mi, nj + 1), order="F"),
               "corr_pres": np.zeros((mi + 1, nj + 1), order="F")}
        lib.ixo_get_aux(self.h, *[_p(out[k]) for k in ("au", "av", "b_o", "Resu", "corr_pres")])
        return out

    def set_corr_pres(self, cp):
        a = np.asfortranarray(cp, dtype=np.float64)
        lib.ixo_set_corr_pres(self.h, _p(a))

    def set_auav(self, au, av):
        a = np.asfortranarray(au, dtype=np.float64)
        b = np.asfortranarray(av, dtype=np.float64)
        lib.ixo_set_auav(self.h, _p(a), _p(b))

    def metric(self, name: str) -> np.ndarray:
        n = {"deltaxp": self.mi, "deltayp": self.nj, "deltaxu": self.mi, "deltayu": self.nj, "deltaxv": self.mi,
             "deltayv": self.nj, "fexp": self.mi, "feyp": self.nj, "fexu": self.mi, "feyv": self.nj, "xu": self.mi,
             "yv": self.nj, "xp": self.mi + 1, "yp": self.nj + 1}[name]
        out = np.zeros(n)
        lib.ixo_get_metric(self.h, METRICS.index(name), _p(out))
        return out

    def _rep(self, r) -> dict:
        d = dict(zip(REPORT_KEYS, list(r)))
        for k in ("n_simple", "n_momen", "n_pres", "n_ener", "exit_code"):
            d[k] = int(d[k])
        return d

    def iterations(self, n: int) -> dict:
        r = (C.c_double * 10)()
        lib.ixo_simple_iterations(self.h, n, r)
        return self._rep(r)

    def loop(self) -> dict:
        r = (C.c_double * 10)()
        lib.ixo_simple_loop(self.h, r)
        return self._rep(r)

    def roll(self):
        lib.ixo_roll(self.h)

    def phase(self, which: int):
        if lib.ixo_phase(self.h, which) != 0:
            raise ValueError(which)

    def nusselt_x(self, j0: int, j1: int):
        T = np.asfortranarray(self.get_state()["T"])
        a, b = C.c_double(), C.c_double()
        if lib.ixo_nusselt_x(self.h, _p(T), j0, j1, C.byref(a), C.byref(b)) != 0:
            raise ValueError("nusselt range")
        return a.value, b.value

    def nusselt_y(self, i0: int, i1: int):
        T = np.asfortranarray(self.get_state()["T"])
        a, b = C.c_double(), C.c_double()
        if lib.ixo_nusselt_y(self.h, _p(T), i0, i1, C.byref(a), C.byref(b)) != 0:
            raise ValueError("nusselt range")
        return a.value, b.value

    def close(self):
        if self.h:
            lib.ixo_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
