"""libixb.so loads and exports every symbol of include/ixb.h; host-side
input logic (boundary-table location, list-directed file parsing).  CPU only:
no compute call needs a GPU here."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from ixchel2d_b200 import _ffi as F
from ixchel2d_b200 import cases

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    txt = (ROOT / "include" / "ixb.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(ixb_\w+)\s*\(", txt, re.M)))


def test_every_declared_symbol_is_exported_and_bound():
    names = _declared()
    assert len(names) >= 25
    raw = C.CDLL(str(F.LIB_PATH))
    for n in names:
        assert hasattr(raw, n), n
    bound = {s[0] for s in F.SIGNATURES}
    assert set(names) == bound


def test_fortran_module_binds_every_declared_function():
    txt = (ROOT / "include" / "mod_ixb.f90").read_text()
    bound = set(re.findall(r'bind\(C,\s*name="(ixb_\w+)"\)', txt))
    assert bound == set(_declared())


def test_strerror_and_version():
    assert F.lib.ixb_version() >= 100
    for s in range(9):
        assert F.lib.ixb_strerror(s)
    assert F.lib.ixb_strerror(0) == b"ok"


def test_create_rejects_bad_sizes():
    h = C.c_void_p()
    assert F.lib.ixb_create(2, 64, 0, C.byref(h)) == F.EINVAL
    assert F.lib.ixb_create(64, 64, 7, C.byref(h)) == F.EINVAL
    assert F.lib.ixb_create(64, 64, 0, None) == F.EINVAL


def test_create_without_gpu_fails_cleanly():
    if F.lib.ixb_device_count() > 0:
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert F.lib.ixb_create(16, 16, 0, C.byref(h)) == F.ECUDA
    assert not h.value


def test_tridiag_status_without_gpu():
    if F.lib.ixb_device_count() > 0:
        pytest.skip("a GPU is present")
    assert F.lib.ixb_tridiag_status() == F.ECUDA


def _locate_ref(coord, x1s, size):
    """lectura_cond_frontera, source/mod_cond_frontera.f90:125-149."""
    idx = [2]
    for x1 in x1s:
        kk = 1
        while kk <= size and not (coord[kk - 1] > x1):
            kk += 1
        idx.append(kk)
    idx[len(x1s)] = size - 1
    return idx


def _lib_locate(side, segs, xx, yy):
    """The library's ixb_bc_locate on the same segments."""
    out = F.BCSide()
    nd = len(segs)
    x1 = (C.c_double * max(nd, 1))(*[s[0] for s in segs])
    ty = (C.c_int * max(nd, 1))(*[s[1] for s in segs])
    va = (C.c_double * max(nd, 1))(*[s[2] for s in segs])
    xx = np.ascontiguousarray(xx, dtype=np.float64)
    yy = np.ascontiguousarray(yy, dtype=np.float64)
    F.check(F.lib.ixb_bc_locate(side, nd, x1, ty, va, F.dptr(xx), xx.size, F.dptr(yy), yy.size, C.byref(out)),
            "ixb_bc_locate")
    return out


@pytest.mark.parametrize("nseg", [0, 1, 5])
@pytest.mark.parametrize("side", [0, 1, 2, 3])
def test_bc_locate_follows_reference_rule(side, nseg):
    c = cases.lid_driven_mixed(31, 19)
    xx, yy = c.xp, c.yp
    coord = yy if side in (0, 2) else xx
    x1s = [0.2, 0.55, 0.1, 0.9, 5.0][:nseg]  # unsorted and past the end on purpose
    segs = [(x, F.BC_DIRI if k % 2 else F.BC_NEUM, float(k)) for k, x in enumerate(x1s)]
    b = _lib_locate(side, segs, xx, yy)
    assert b.ndivis == nseg and b.side == side
    assert list(b.index[:nseg + 1]) == _locate_ref(coord, x1s, coord.size)
    assert list(b.type[:nseg]) == [s[1] for s in segs]
    assert list(b.value[:nseg]) == [s[2] for s in segs]
    # the case builders' table (built without the library) is the same table, byte for byte
    p = cases.bc_side(side, segs, xx, yy)
    assert bytes(p) == bytes(b)


def test_read_bc_file(tmp_path):
    c = cases.natural_cavity(12, 10)
    f = tmp_path / "cond_fronterat.dat"
    # list-directed records: comments after the values are discarded, D exponents accepted
    f.write_text(
        "temp a 1   ! lado izquierdo\n"
        "0.0 1.0D+00 diri 1.0D0\n"
        "temp c 1\n"
        "0.0, 1.0, diri, 0.0\n"
        "'temp' 'b' 2\n"
        "0.0 0.4 neum 0.0\n"
        "0.4 1.0 diri 0.25\n"
        "temp d 1\n"
        "0.0 1.0 neum 0.0 extra ignored\n")
    out = (F.BCSide * 4)()
    xx, yy = c.xp, c.yp
    st = F.lib.ixb_read_bc_file(str(f).encode(), F.dptr(xx), xx.size, F.dptr(yy), yy.size, out)
    assert st == F.OK
    a, b, cc, d = out
    assert a.ndivis == 1 and a.type[0] == F.BC_DIRI and a.value[0] == 1.0 and list(a.index[:2]) == [2, 10]
    assert cc.ndivis == 1 and cc.type[0] == F.BC_DIRI and cc.value[0] == 0.0
    assert b.ndivis == 2 and list(b.type[:2]) == [F.BC_NEUM, F.BC_DIRI] and b.value[1] == 0.25
    assert list(b.index[:3]) == _locate_ref(xx, [0.4, 1.0], xx.size)
    assert d.ndivis == 1 and d.type[0] == F.BC_NEUM


def test_read_bc_file_missing(tmp_path):
    out = (F.BCSide * 4)()
    x = np.linspace(0, 1, 5)
    assert F.lib.ixb_read_bc_file(str(tmp_path / "nope.dat").encode(), F.dptr(x), 5, F.dptr(x), 5, out) == F.EIO


def test_mesh_builder_matches_malla_irr_uniform():
    xu, yv, xp, yp = cases.staggered_mesh(9, 7)
    assert np.allclose(xu, np.arange(9) / 8.0, rtol=0, atol=1e-15)
    assert xp[0] == pytest.approx(-1 / 16) and xp[-1] == pytest.approx(1 + 1 / 16)
    assert np.allclose(xp[1:-1], (xu[1:] + xu[:-1]) / 2, rtol=1e-14)
