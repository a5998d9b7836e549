"""Mesh generation and the D23.15 mesh/state files (host only, no GPU)."""
import ctypes as C
import math

import numpy as np
import pytest

from ixchel2d_b200 import _ffi as F
from ixchel2d_b200 import cases


def _axis(kind, n, length=1.0, param=1.2, centre=0.5):
    out = np.zeros(n)
    assert F.lib.ixb_mesh_axis(kind, n, length, param, centre, F.dptr(out)) == F.OK
    return out


@pytest.mark.parametrize("kind,name", [(F.MESH_UNIF, "unif"), (F.MESH_TUBO, "tubo"), (F.MESH_CENT, "cent"),
                                       (F.MESH_TANH, "tanh")])
def test_axis_matches_the_python_restatement(kind, name):
    for n in (5, 64, 301):
        a = _axis(kind, n, 2.0, 1.7, 1.0)
        b = cases.axis_nodes(name, n, 2.0, 1.7, 1.0)
        assert np.allclose(a, b, rtol=0, atol=1e-15 * 2.0), (name, n)
        assert np.all(np.diff(a) > 0)
        assert abs(a[0]) < 1e-14 and abs(a[-1] - 2.0) < 1e-13


def test_tanh_clusters_at_both_walls():
    x = _axis(F.MESH_TANH, 101, 1.0, 1.2)
    d = np.diff(x)
    assert d[0] < d[50] and d[-1] < d[50]
    assert np.allclose(d, d[::-1], rtol=1e-12)


def test_staggered_mesh_matches_cases():
    mi, nj = 37, 23
    xu, yv, xp, yp = np.zeros(mi), np.zeros(nj), np.zeros(mi + 1), np.zeros(nj + 1)
    st = F.lib.ixb_staggered_mesh(mi, nj, F.MESH_TANH, 1.2, F.MESH_UNIF, 1.2, 1.0, 1.0,
                                  *map(F.dptr, (xu, yv, xp, yp)))
    assert st == F.OK
    ref = cases.staggered_mesh(mi, nj, "tanh", "unif", xparam=1.2, yparam=1.2)
    for a, b in zip((xu, yv, xp, yp), ref):
        # libm's tanh and numpy's may differ in the last bits; both are then
        # rounded to 15 significant digits (one unit of the 15th digit apart)
        assert np.allclose(a, b, rtol=0, atol=2.1e-15), np.max(np.abs(a - b))
    # p nodes: one half cell outside each wall
    assert xp[0] < 0 < xp[1] and xp[-1] > 1.0


def _fields(mi, nj, seed=3):
    rng = np.random.default_rng(seed)
    f = lambda *s: np.asfortranarray(rng.standard_normal(s) * 10.0 ** rng.integers(-120, 120, s))
    return f(mi, nj + 1), f(mi + 1, nj), f(mi + 1, nj + 1), f(mi + 1, nj + 1)


def test_state_files_round_trip(tmp_path):
    mi, nj = 9, 7
    xu, yv, xp, yp = cases.staggered_mesh(mi, nj, "tubo", "cent")
    u, v, T, p = _fields(mi, nj)
    names = [str(tmp_path / f"{k}.dat").encode() for k in "uvp"]
    st = F.lib.ixb_write_state_files(*names, mi, nj, *map(F.dptr, (xu, yv, xp, yp, u, v, T, p)), 3, 40, 1000, 1.0)
    assert st == F.OK
    out = [np.zeros_like(a) for a in (xu, yv, xp, yp)] + [np.zeros_like(a, order="F") for a in (u, v, T, p)]
    i0, i1, it, a = C.c_int(), C.c_int(), C.c_int(), C.c_double()
    st = F.lib.ixb_read_state_files(*names, mi, nj, *map(F.dptr, out), C.byref(i0), C.byref(i1), C.byref(it),
                                    C.byref(a))
    assert st == F.OK and (i0.value, i1.value, it.value, a.value) == (3, 40, 1000, 1.0)
    for got, want in zip(out, (xu, yv, xp, yp, u, v, T, p)):
        # D23.15 keeps 15 significant digits
        assert np.allclose(got, want, rtol=1e-14, atol=0), np.max(np.abs(got - want) / np.abs(want))
    # the records are Fortran D23.15: 23 characters, a D exponent below |e| = 100
    line = open(names[0], "r").read().splitlines()[1]
    assert len(line) == 69 and line[22] in "0123456789"
    first = line[:23].strip()
    assert first.startswith(("0.", "-0.")) and ("D" in first or first[-4] in "+-")


def test_fortran_d_exponents_are_read(tmp_path):
    # a record as the reference writes it, including a three-digit exponent
    mi, nj = 2, 2
    lines = [" 1 2 0 0.1D+01"]
    for jj in range(nj + 1):
        for ii in range(mi):
            lines.append(f"  0.{ii + 1}00000000000000D+01  0.{jj + 1}00000000000000D+01 -0.250000000000000-120")
    (tmp_path / "u.dat").write_text("\n".join(lines) + "\n")
    xu, yv, xp, yp = cases.staggered_mesh(mi, nj)
    u, v, T, p = _fields(mi, nj)
    names = [str(tmp_path / f"{k}.dat").encode() for k in "uvp"]
    assert F.lib.ixb_write_state_files(names[1], names[1], names[2], mi, nj,
                                       *map(F.dptr, (xu, yv, xp, yp, u, v, T, p)), 1, 2, 0, 1.0) == F.OK
    out = [np.zeros_like(a) for a in (xu, yv, xp, yp)] + [np.zeros_like(a, order="F") for a in (u, v, T, p)]
    st = F.lib.ixb_read_state_files(*names, mi, nj, *map(F.dptr, out), None, None, None, None)
    assert st == F.OK
    assert np.all(out[4] == -0.25e-120)
    assert out[0][1] == 2.0


def test_missing_file_is_an_io_error(tmp_path):
    mi, nj = 4, 4
    bufs = [np.zeros(s) for s in (mi, nj, mi + 1, nj + 1)] + [np.zeros((mi + 1) * (nj + 1))] * 4
    nope = str(tmp_path / "nope.dat").encode()
    assert F.lib.ixb_read_state_files(nope, nope, nope, mi, nj, *map(F.dptr, bufs), None, None, None, None) == F.EIO
