"""Python view of one libixb handle: the SIMPLE hot path of Ixchel2D on one
GPU, driven through the C ABI (include/ixb.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi as F
from .cases import Case, shapes


def _f64(a) -> np.ndarray:
    return np.asfortranarray(a, dtype=np.float64)


class Simple2D:
    """Owns an ixb handle (device memory + stream) for an (mi, nj) grid."""

    def __init__(self, mi: int, nj: int, prec: int = F.PREC_FP64, handle=None):
        self.mi, self.nj = mi, nj
        if handle is None:
            h = C.c_void_p()
            F.check(F.lib.ixb_create(mi, nj, prec, C.byref(h)), "ixb_create")
            self._owned = True
        else:  # a handle owned elsewhere (an instance of a batch)
            h = handle
            self._owned = False
        self.h = h
        self._shapes = shapes(mi, nj)

    def setup(self, case: Case, **param_over) -> "Simple2D":
        """Mesh, parameters, boundary tables, sources and state of `case`."""
        self.set_mesh(case.xu, case.yv, case.xp, case.yp)
        prm = dict(case.params)
        prm.update(param_over)
        self.set_params(**prm)
        for var, sides in case.bc.items():
            self.set_bc(var, sides)
        for var, (fc, fl) in case.sources.items():
            self.set_sources(var, fc, fl)
        self.upload(case.state)
        return self

    # ---- setup ----
    def set_mesh(self, xu, yv, xp, yp):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (xu, yv, xp, yp)]
        F.check(F.lib.ixb_set_mesh(self.h, *map(F.dptr, arrs)), "ixb_set_mesh")

    def set_params(self, **kw):
        p = F.Params()
        for k, v in kw.items():
            setattr(p, k, v)
        F.check(F.lib.ixb_set_params(self.h, C.byref(p)), "ixb_set_params")

    def set_bc(self, var: int, sides):
        arr = (F.BCSide * 4)(*sides)
        F.check(F.lib.ixb_set_bc(self.h, var, arr), "ixb_set_bc")

    def set_sources(self, var: int, fcon=None, flin=None):
        fc = None if fcon is None else _f64(fcon)
        fl = None if flin is None else _f64(flin)
        F.check(F.lib.ixb_set_sources(self.h, var, F.dptr(fc), F.dptr(fl)), "ixb_set_sources")

    def upload(self, state: dict):
        keys = ("u", "v", "p", "T", "u_ant", "v_ant", "T_ant")
        arrs = [None if state.get(k) is None else _f64(state[k]) for k in keys]
        for k, a in zip(keys, arrs):
            if a is not None and a.shape != self._shapes[k]:
                raise ValueError(f"{k}: shape {a.shape} != {self._shapes[k]}")
        F.check(F.lib.ixb_upload_state(self.h, *map(F.dptr, arrs)), "ixb_upload_state")

    def download(self, out: dict | None = None) -> dict:
        """The seven state arrays; with `out`, written into its arrays (float64,
        Fortran-ordered, the reference's shapes; e.g. views of pinned memory,
        which the copies then reach directly) instead of new ones."""
        keys = ("u", "v", "p", "T", "u_ant", "v_ant", "T_ant")
        if out is None:
            out = {k: np.empty(s, order="F") for k, s in self._shapes.items()}
        else:
            for k in keys:
                a = out[k]
                if a.dtype != np.float64 or not a.flags.f_contiguous or a.shape != self._shapes[k]:
                    raise ValueError(f"{k}: needs a float64 Fortran-ordered array of shape {self._shapes[k]}")
        F.check(F.lib.ixb_download_state(self.h, *[F.dptr(out[k]) for k in keys]), "ixb_download_state")
        return out

    def download_aux(self) -> dict:
        mi, nj = self.mi, self.nj
        out = {"au": np.zeros((mi, nj + 1), order="F"), "av": np.zeros((mi + 1, nj), order="F"),
               "b_o": np.zeros((mi + 1, nj + 1), order="F"), "Resu": np.zeros((mi, nj + 1), order="F"),
               "corr_pres": np.zeros((mi + 1, nj + 1), order="F")}
        F.check(F.lib.ixb_download_aux(self.h, *[F.dptr(out[k]) for k in ("au", "av", "b_o", "Resu", "corr_pres")]),
                "ixb_download_aux")
        return out

    def set_work(self, corr_pres=None, au=None, av=None):
        a = [None if x is None else _f64(x) for x in (corr_pres, au, av)]
        F.check(F.lib.ixb_set_work(self.h, *map(F.dptr, a)), "ixb_set_work")

    @classmethod
    def from_case(cls, case: Case, prec: int = F.PREC_FP64, **param_over) -> "Simple2D":
        return cls(case.mi, case.nj, prec).setup(case, **param_over)

    # ---- hot path ----
    def iterations(self, n: int) -> dict:
        r = F.Report()
        F.check(F.lib.ixb_simple_iterations(self.h, n, C.byref(r)), "ixb_simple_iterations")
        return r.as_dict()

    def loop(self) -> dict:
        r = F.Report()
        F.check(F.lib.ixb_simple_loop(self.h, C.byref(r)), "ixb_simple_loop")
        return r.as_dict()

    def converge(self, k0: int, k1: int, vertical: bool = True, wall: int = 0, every: int = 1000,
                 tol_dnu: float = 1e-8, tol_maxbo: float = 0.0, max_iters: int = 200000) -> dict:
        """Outer iterations until the monitored wall's Nusselt number changes by
        less than tol_dnu between evaluations `every` iterations apart (exit_code
        3), maxbo < tol_maxbo (4) or max_iters (5), all on the device in one
        graph launch (ixb_simple_converge).  The report adds 'nu' (both walls at
        the last evaluation) and 'dnu' (the monitored wall's last change)."""
        m = F.NuMonitor(vertical=int(vertical), k0=k0, k1=k1, wall=wall, every=every, reserved=0,
                        max_iters=max_iters, tol_dnu=tol_dnu, tol_maxbo=tol_maxbo)
        r = F.Report()
        nu = np.zeros(2)
        dnu = C.c_double()
        F.check(F.lib.ixb_simple_converge(self.h, C.byref(m), C.byref(r), F.dptr(nu), C.byref(dnu)),
                "ixb_simple_converge")
        out = r.as_dict()
        out["nu"] = (float(nu[0]), float(nu[1]))
        out["dnu"] = dnu.value
        return out

    def step(self) -> dict:
        r = F.Report()
        F.check(F.lib.ixb_step(self.h, C.byref(r)), "ixb_step")
        return r.as_dict()

    def roll(self):
        F.check(F.lib.ixb_roll(self.h), "ixb_roll")

    def phase(self, which: int):
        F.check(F.lib.ixb_phase(self.h, which), "ixb_phase")

    def time_phases(self, reps: int = 20, flush_bytes: int = 0) -> list[float]:
        """Mean device milliseconds per launch of each phase 0..9 (advances the state);
        flush_bytes > 0 writes that many bytes before every launch (cold L2)."""
        ms = np.zeros(10)
        F.check(F.lib.ixb_time_phases(self.h, reps, flush_bytes, F.dptr(ms)), "ixb_time_phases")
        return ms.tolist()

    def nusselt_x(self, j0: int, j1: int):
        a, b = C.c_double(), C.c_double()
        F.check(F.lib.ixb_nusselt_x(self.h, j0, j1, C.byref(a), C.byref(b)), "ixb_nusselt_x")
        return a.value, b.value

    def nusselt_y(self, i0: int, i1: int):
        a, b = C.c_double(), C.c_double()
        F.check(F.lib.ixb_nusselt_y(self.h, i0, i1, C.byref(a), C.byref(b)), "ixb_nusselt_y")
        return a.value, b.value

    SHAPES = ((1, 128), (1, 256), (1, 512), (2, 64), (2, 128), (4, 32), (4, 64), (4, 128), (5, 64), (5, 128),
              (6, 64), (6, 128), (8, 32), (8, 64), (8, 128), (16, 16), (16, 32))

    def set_sweep_shape(self, sweep: int, lines_per_cta: int = 0, threads_per_line: int = 0):
        F.check(F.lib.ixb_set_sweep_shape(self.h, sweep, lines_per_cta, threads_per_line), "ixb_set_sweep_shape")

    def iteration_launches(self) -> int:
        """Kernels one outer iteration launches with the current shapes (one inner pass per loop)."""
        k = C.c_int()
        F.check(F.lib.ixb_iteration_launches(self.h, C.byref(k)), "ixb_iteration_launches")
        return k.value

    def autotune(self, reps: int = 5, flush_bytes: int = 0) -> dict:
        """Pick the fastest launch shape of every sweep; returns {sweep: (lines_per_cta, threads_per_line, ms)}."""
        chosen = (C.c_int * 16)()
        ms = np.zeros(8)
        F.check(F.lib.ixb_autotune(self.h, reps, flush_bytes, chosen, F.dptr(ms)), "ixb_autotune")
        return {k: (chosen[2 * k], chosen[2 * k + 1], float(ms[k])) for k in range(8)}

    # ---- energy equation with the flow fixed, and its adjoint ----
    def energy_iterations(self, n: int):
        F.check(F.lib.ixb_energy_iterations(self.h, n), "ixb_energy_iterations")

    def adjoint_energy(self, K: int, j0: int, j1: int) -> np.ndarray:
        """d nu0(ixb_nusselt_x(j0, j1)) / d (side-a value of T x-line jj), jj = 1..nj+1, after K passes."""
        g = np.zeros(self.nj + 1)
        F.check(F.lib.ixb_adjoint_energy(self.h, K, j0, j1, F.dptr(g)), "ixb_adjoint_energy")
        return g

    def adjoint_energy_coupled(self, K: int, ckpt: int, j0: int, j1: int):
        """(grad, nu0) after K outer iterations from the current state, for a flow that does not depend on T
        (Ri = Riy = 0): grad[jj-1] = d nu0 / d (side-a value of T x-line jj); checkpoints every ckpt iterations.
        Leaves the state after the K iterations."""
        g = np.zeros(self.nj + 1)
        nu = C.c_double()
        F.check(F.lib.ixb_adjoint_energy_coupled(self.h, K, ckpt, j0, j1, F.dptr(g), C.byref(nu)),
                "ixb_adjoint_energy_coupled")
        return g, nu.value

    def adjoint_simple(self, K: int, ckpt: int, j0: int, j1: int, gradient: bool = True):
        """Hot-wall Nusselt number nu0 after K outer iterations (one pass of each
        equation) and, with `gradient`, its gradient with respect to the side-a
        T boundary value of every x-line (nj+1 entries) through the full coupled
        iteration (ixb_adjoint_simple).  Returns (grad or None, nu0)."""
        g = np.zeros(self.nj + 1) if gradient else None
        nu = C.c_double()
        F.check(F.lib.ixb_adjoint_simple(self.h, K, ckpt, j0, j1, None if g is None else g.ctypes.data,
                                         C.addressof(nu)), "ixb_adjoint_simple")
        return g, nu.value

    def set_bc_values(self, var: int, side: int, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        F.check(F.lib.ixb_set_bc_values(self.h, var, side, F.dptr(v)), "ixb_set_bc_values")

    def set_stream(self, stream_handle: int):
        """Launch on an external cudaStream_t (e.g. torch.cuda.Stream().cuda_stream)."""
        F.check(F.lib.ixb_set_stream(self.h, C.c_void_p(stream_handle)), "ixb_set_stream")

    def close(self):
        if getattr(self, "h", None):
            if self._owned:
                F.lib.ixb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
