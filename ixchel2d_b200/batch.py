"""Python view of a libixb batch: many SIMPLE instances (cavities of
different sizes and parameters) advanced together, one launch per phase for
all of them (ixb_batch_* in include/ixb.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _ffi as F
from .cases import Case
from .simple import Simple2D


class Batch:
    """Owns an ixb batch; instance i is reachable as a (non-owning) Simple2D."""

    def __init__(self, sizes, prec: int = F.PREC_FP32_REFINED):
        sizes = [(int(m), int(n)) for m, n in sizes]
        mi = (C.c_int * len(sizes))(*[m for m, _ in sizes])
        nj = (C.c_int * len(sizes))(*[n for _, n in sizes])
        b = C.c_void_p()
        F.check(F.lib.ixb_batch_create(len(sizes), mi, nj, prec, C.byref(b)), "ixb_batch_create")
        self.b = b
        self.count = len(sizes)
        self.instances = []
        for i, (m, n) in enumerate(sizes):
            h = C.c_void_p()
            F.check(F.lib.ixb_batch_instance(b, i, C.byref(h)), "ixb_batch_instance")
            self.instances.append(Simple2D(m, n, handle=h))

    @classmethod
    def from_cases(cls, cases: list[Case], prec: int = F.PREC_FP32_REFINED, **param_over) -> "Batch":
        bt = cls([(c.mi, c.nj) for c in cases], prec)
        for inst, case in zip(bt.instances, cases):
            inst.setup(case, **param_over)
        bt.restart()
        return bt

    def __getitem__(self, i: int) -> Simple2D:
        return self.instances[i]

    def restart(self):
        F.check(F.lib.ixb_batch_restart(self.b), "ixb_batch_restart")

    def iterate(self, max_iters: int) -> int:
        """Up to max_iters outer iterations of the active instances; returns how many remain active."""
        n = C.c_int()
        F.check(F.lib.ixb_batch_iterate(self.b, max_iters, C.byref(n)), "ixb_batch_iterate")
        return n.value

    def report(self, i: int) -> dict:
        r = F.Report()
        F.check(F.lib.ixb_batch_report(self.b, i, C.byref(r)), "ixb_batch_report")
        return r.as_dict()

    def set_sweep_shape(self, sweep: int, lines_per_cta: int = 0, threads_per_line: int = 0):
        F.check(F.lib.ixb_batch_set_sweep_shape(self.b, sweep, lines_per_cta, threads_per_line),
                "ixb_batch_set_sweep_shape")

    def autotune(self, reps: int = 3) -> dict:
        chosen = (C.c_int * 16)()
        ms = (C.c_double * 8)()
        F.check(F.lib.ixb_batch_autotune(self.b, reps, chosen, ms), "ixb_batch_autotune")
        return {k: (chosen[2 * k], chosen[2 * k + 1], float(ms[k])) for k in range(8)}

    def close(self):
        if getattr(self, "b", None):
            for inst in self.instances:
                inst.h = None
            F.lib.ixb_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
