"""The FP32 + FP64-refined form (IXB_PREC_FP32_REFINED) against the binary64
path and the oracle, at convergence.

The mixed form solves every line in binary32 (u, v and T as binary64
defect corrections, p' outright), so its fields after a fixed number of
iterations are not within 1e-10 of the binary64 ones; what it must give is
the same converged answer:
the hot-wall Nusselt number within 1e-6 of the binary64 oracle's, with the
mass residual driven below 1e-8 and the fields' relative L2 distance stated
and bounded.
"""
import numpy as np
import pytest

from ixchel2d_b200 import _ffi as F
from ixchel2d_b200 import cases
from ixchel2d_b200.simple import Simple2D
from oracle.oracle import OracleCase as _OracleCase

pytestmark = pytest.mark.gpu

STATE = ("u", "v", "p", "T")
DNU_TOL = 1e-6     # |Nu(mixed) - Nu(binary64 oracle)| at convergence
FIELD_TOL = 1e-5   # relative L2 distance of u, v, T to the binary64 oracle at convergence
MAXBO_TOL = 1e-8   # mass residual the converged run must reach


@pytest.fixture(autouse=True)
def _need_gpu():
    if F.lib.ixb_device_count() < 1:
        pytest.skip("no CUDA device")


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _converge(g, chunk, cap):
    it, rep = 0, None
    while it < cap:
        rep = g.iterations(chunk)
        it += chunk
        if rep["maxbo"] < MAXBO_TOL:
            break
    return it, rep


def test_refined_natural_cavity_converges_to_the_binary64_nusselt():
    # the plain small configuration: 64x64, Ra=1e4, Pr=0.71, T0=0.5
    case = cases.natural_cavity(64, 64, Ra=1e4, T0=0.5)
    g = Simple2D.from_case(case, prec=F.PREC_FP32_REFINED)
    it, rep = _converge(g, 200, 20000)
    assert rep["maxbo"] < MAXBO_TOL, rep
    o = _OracleCase(case)
    o.iterations(it)
    gs, os_ = g.download(), o.get_state()
    ng, no = g.nusselt_x(2, 62), o.nusselt_x(2, 62)
    assert abs(ng[0] - no[0]) < DNU_TOL and abs(ng[1] - no[1]) < DNU_TOL, (ng, no)
    for k in ("u", "v", "T"):
        assert rel_l2(gs[k], os_[k]) < FIELD_TOL, (k, rel_l2(gs[k], os_[k]))


def test_refined_lid_driven_tanh_converges_to_the_binary64_nusselt():
    # the mixed-convection heated lid on a tanh mesh, reduced in size
    case = cases.lid_driven_mixed(91, 61)
    g64 = Simple2D.from_case(case)
    g32 = Simple2D.from_case(case, prec=F.PREC_FP32_REFINED)
    it64, r64 = _converge(g64, 200, 40000)
    it32, r32 = _converge(g32, 200, 40000)
    assert r64["maxbo"] < MAXBO_TOL and r32["maxbo"] < MAXBO_TOL, (r64, r32)
    n64, n32 = g64.nusselt_y(2, 89), g32.nusselt_y(2, 89)
    assert abs(n64[0] - n32[0]) < DNU_TOL and abs(n64[1] - n32[1]) < DNU_TOL, (n64, n32)
    s64, s32 = g64.download(), g32.download()
    for k in ("u", "v", "T"):
        assert rel_l2(s32[k], s64[k]) < FIELD_TOL, (k, rel_l2(s32[k], s64[k]))


@pytest.mark.parametrize("shape", Simple2D.SHAPES)
def test_refined_every_launch_shape(shape):
    case = cases.lid_driven_mixed(45, 29)
    ref = Simple2D.from_case(case, prec=F.PREC_FP32_REFINED)
    g = Simple2D.from_case(case, prec=F.PREC_FP32_REFINED)
    for k in range(8):
        g.set_sweep_shape(k, *shape)
    ref.iterations(60)
    g.iterations(60)
    a, b = g.download(), ref.download()
    for k in STATE:
        assert np.all(np.isfinite(a[k])), k
        # different partitions of the binary32 line solve round differently
        assert rel_l2(a[k], b[k]) < 1e-4, (k, rel_l2(a[k], b[k]))


def test_refined_early_iterations_track_binary64():
    # before convergence the two forms differ by binary32 rounding only
    case = cases.natural_cavity(40, 36, Ra=1e5)
    g = Simple2D.from_case(case, prec=F.PREC_FP32_REFINED)
    o = _OracleCase(case)
    g.iterations(50)
    o.iterations(50)
    gs, os_ = g.download(), o.get_state()
    for k in ("u", "v", "T"):
        assert rel_l2(gs[k], os_[k]) < 1e-4, (k, rel_l2(gs[k], os_[k]))


def test_refined_exact_solver_ignores_the_mode():
    # IXB_SOLVER_EXACT runs the binary64 reference order in either mode
    case = cases.lid_driven_mixed(37, 23)
    g = Simple2D.from_case(case, prec=F.PREC_FP32_REFINED, solver=F.SOLVER_EXACT)
    o = _OracleCase(case)
    g.iterations(30)
    o.iterations(30)
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert np.array_equal(gs[k], os_[k]), k


def test_refined_immersed_body_penalties():
    # an immersed block with the penalty sources of definir_cuerpo
    # ('chime', mod_front_inmersa.f90:150-167): ~1e51 on the u, v and T
    # diagonals, beyond the binary32 range
    case = cases.natural_cavity(32, 32, Ra=1e4)
    mi, nj = case.mi, case.nj
    fu = np.zeros((mi, nj + 1), order="F"); lu = np.zeros_like(fu)
    fv = np.zeros((mi + 1, nj), order="F"); lv = np.zeros_like(fv)
    ft = np.zeros((mi + 1, nj + 1), order="F"); lt = np.zeros_like(ft)
    for f, l in ((fu, lu), (fv, lv)):
        f[12:18, 12:18] = 10.0e50 * 10.0e-12
        l[12:18, 12:18] = -10.0e50
    ft[12:18, 12:18] = 10e50 * 0.5
    lt[12:18, 12:18] = -10e50
    case.sources = {0: (fu, lu), 1: (fv, lv), 2: (ft, lt)}
    g32 = Simple2D.from_case(case, prec=F.PREC_FP32_REFINED)
    g64 = Simple2D.from_case(case)
    g32.iterations(200)
    g64.iterations(200)
    a, b = g32.download(), g64.download()
    for k in ("u", "v", "T"):
        assert np.all(np.isfinite(a[k])), k
        assert rel_l2(a[k], b[k]) < 1e-4, (k, rel_l2(a[k], b[k]))
    # the block holds T = fcon / -flin = 0.5
    assert np.allclose(a["T"][13:17, 13:17], 0.5, atol=1e-9)
