"""Immersed solid bodies as penalty sources (ixb_body_sources, host only):
the library's masks against the oracle's loop-by-loop restatement of
definir_cuerpo (source/mod_front_inmersa.f90:54-179)."""
import numpy as np
import pytest

from ixchel2d_b200 import _ffi as F
from ixchel2d_b200 import cases
from oracle import oracle as O


def _case(mi, nj, ao=10.0, bo=1.0, xkind="tubo"):
    """A case on [0, ao] x [0, bo], where the reference's fixed bodies lie."""
    case = cases.natural_cavity(8, 8)
    xu, yv, xp, yp = cases.staggered_mesh(mi, nj, xkind, "unif", ao=ao, bo=bo)
    case.mi, case.nj, case.xu, case.yv, case.xp, case.yp = mi, nj, xu, yv, xp, yp
    case.sources = {}
    return case


@pytest.mark.parametrize("shape,name", [(F.BODY_TRIAN, "trian"), (F.BODY_CUADR, "cuadr"), (F.BODY_CHIME, "chime")])
@pytest.mark.parametrize("mi,nj", [(120, 40), (301, 97)])
def test_fixed_shapes_match_the_oracle(shape, name, mi, nj):
    case = cases.add_body(_case(mi, nj, xkind="unif"), shape)
    ref = O.definir_cuerpo(name, mi, nj, case.xp, case.yp)
    hit = 0
    for var in (0, 1, 2):
        f, l = case.sources.get(var, (np.zeros_like(ref[var][0]), np.zeros_like(ref[var][1])))
        assert np.array_equal(f, ref[var][0]), (name, var)
        assert np.array_equal(l, ref[var][1]), (name, var)
        hit += int(np.count_nonzero(l))
    assert hit > 0, name  # the body covers some nodes of this mesh


def test_general_forms_reproduce_the_fixed_shapes():
    mi, nj = 150, 60
    box = cases.add_body(_case(mi, nj), F.BODY_BOX, [6.0 - 0.1 / 2.0, 6.0 + 0.1 / 2.0, 0.05 - 0.1 / 2.0,
                                                     0.05 + 0.1 / 2.0], F.BODY_VEL)
    cuadr = cases.add_body(_case(mi, nj), F.BODY_CUADR)
    b1 = -(0.1 - 0.5 * 6.0) / 0.5
    b2 = -(0.1 - (-0.5) * 6.0) / (-0.5)
    region = cases.add_body(_case(mi, nj), F.BODY_REGION, [0.0, 0.1, 2.0, b1, -2.0, b2], F.BODY_VEL)
    trian = cases.add_body(_case(mi, nj), F.BODY_TRIAN)
    for a, b in ((box, cuadr), (region, trian)):
        for var in (0, 1):
            assert np.array_equal(a.sources[var][0], b.sources[var][0])
            assert np.array_equal(a.sources[var][1], b.sources[var][1])
            assert np.count_nonzero(a.sources[var][1]) > 0


def test_out_of_range_nodes_and_accumulation():
    mi, nj = 40, 30
    case = _case(mi, nj, ao=1.0, bo=1.0, xkind="unif")
    # a box over the last p column (ii = mi+1, beyond the last u node) and
    # the top p row (jj = nj+1, beyond the last v node)
    cases.add_body(case, F.BODY_BOX, [0.9, 2.0, 0.9, 2.0], F.BODY_VEL | F.BODY_TEMP, 0.25)
    fu, lu = case.sources[0]
    fv, lv = case.sources[1]
    ft, lt = case.sources[2]
    assert lu.shape == (mi, nj + 1) and lv.shape == (mi + 1, nj)
    inside = lambda x, y: 0.9 <= x <= 2.0 and 0.9 <= y <= 2.0
    for jj in range(nj + 1):
        for ii in range(mi + 1):
            on = inside(case.xp[ii], case.yp[jj])
            assert (lt[ii, jj] == -1e51) == on and (ft[ii, jj] == 1e51 * 0.25) == on
            if ii < mi:
                assert (lu[ii, jj] != 0) == on
            if jj < nj:
                assert (lv[ii, jj] != 0) == on
    assert lt[mi, nj] == -1e51  # the corner p node is inside; u and v have no entry there
    # a second body adds to the first
    n0 = np.count_nonzero(lt)
    cases.add_body(case, F.BODY_BOX, [0.0, 0.1, 0.0, 0.1], F.BODY_TEMP, 1.0)
    assert np.count_nonzero(case.sources[2][1]) > n0
    assert np.count_nonzero(case.sources[0][1]) == np.count_nonzero(lu)


def test_bad_arguments():
    xp = np.zeros(11)
    yp = np.zeros(11)
    z = np.zeros(121)  # T arrays: (mi+1)(nj+1)
    assert F.lib.ixb_body_sources(10, 10, F.dptr(xp), F.dptr(yp), 9, None, 0, 0.0, *([None] * 6)) == F.EINVAL
    assert F.lib.ixb_body_sources(10, 10, F.dptr(xp), F.dptr(yp), F.BODY_BOX, None, 0, 0.0,
                                  *([None] * 6)) == F.EINVAL
    prm = np.array([0.0, 1.0, 0.0, 1.0])
    assert F.lib.ixb_body_sources(10, 10, F.dptr(xp), F.dptr(yp), F.BODY_BOX, F.dptr(prm), F.BODY_TEMP, 0.0,
                                  *([None] * 6)) == F.EINVAL
    assert F.lib.ixb_body_sources(10, 10, F.dptr(xp), F.dptr(yp), F.BODY_BOX, F.dptr(prm), F.BODY_TEMP, 0.0,
                                  None, None, None, None, F.dptr(z), F.dptr(np.zeros(121))) == F.OK
    assert np.all(z == 0.0)  # t_value 0: the constant source is 1e51 * 0
