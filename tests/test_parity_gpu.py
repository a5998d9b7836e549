"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances:
* IXB_SOLVER_EXACT: bit-identical (assembly follows the reference operands
  in IEEE order without FMA contraction; Thomas in the reference order).
* IXB_SOLVER_HYBRID (default): the warp Thomas-PCR line solve rounds
  differently, fields agree to 1e-10 relative after N outer iterations.
"""
import ctypes as C
import os

import numpy as np
import pytest

from ixchel2d_b200 import Simple2D, IxbError, cases
from ixchel2d_b200 import _ffi as F
from oracle import oracle as O
from tests.conftest import relerr

pytestmark = pytest.mark.gpu

STATE = ("u", "v", "p", "T", "u_ant", "v_ant", "T_ant")
HYBRID_TOL = 1e-10


@pytest.fixture(autouse=True)
def _need_gpu(has_gpu):
    if not has_gpu:
        pytest.skip("no CUDA device")


def _pair(case, **over):
    g = Simple2D.from_case(case, **over)
    o = O.OracleCase(case, **over)
    return g, o


def _warm_state(case, n=25):
    """A non-trivial state: the oracle's fields after n iterations."""
    o = O.OracleCase(case)
    o.iterations(n)
    return o.get_state(), o.get_aux()


CASES = {
    "natural_24x20": lambda: cases.natural_cavity(24, 20, Ra=1e5),
    "lid_tanh_37x23": lambda: cases.lid_driven_mixed(37, 23, Re=100.0, Ri=1.0),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("phase", list(range(10)))
def test_each_phase_bit_identical(name, phase):
    case = CASES[name]()
    st, aux = _warm_state(case)
    case.state = st
    g, o = _pair(case, solver=F.SOLVER_EXACT)
    # same p', au, av on both sides (phases 4-6 read them)
    rng = np.random.default_rng(phase)
    cp = aux["corr_pres"] + 1e-3 * rng.standard_normal(aux["corr_pres"].shape)
    g.set_work(cp, aux["au"], aux["av"])
    o.set_corr_pres(cp)
    o.set_auav(aux["au"], aux["av"])
    g.phase(phase)
    o.phase(phase)
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert np.array_equal(gs[k], os_[k]), (k, relerr(gs[k], os_[k]))
    ga, oa = g.download_aux(), o.get_aux()
    check = {1: ["au"], 3: ["av"], 4: ["corr_pres"], 5: ["corr_pres", "b_o"], 9: ["Resu"]}.get(phase, [])
    for k in check:
        if k == "b_o" or k == "Resu":
            sl = (slice(1, -1), slice(1, -1))
            assert np.array_equal(ga[k][sl], oa[k][sl]), (k, relerr(ga[k], oa[k]))
        else:
            assert np.array_equal(ga[k], oa[k]), (k, relerr(ga[k], oa[k]))


@pytest.mark.parametrize("name", list(CASES))
def test_iterations_exact_solver_bit_identical(name):
    case = CASES[name]()
    g, o = _pair(case, solver=F.SOLVER_EXACT)
    rg = g.iterations(40)
    ro = o.iterations(40)
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert np.array_equal(gs[k], os_[k]), (k, relerr(gs[k], os_[k]))
    for k in ("maxbo", "residuo", "err_u", "err_p", "err_t"):
        assert abs(rg[k] - ro[k]) <= 1e-12 * abs(ro[k]), k
    assert rg["n_simple"] == 40 and rg["n_momen"] == 40


@pytest.mark.parametrize("name", list(CASES))
def test_iterations_hybrid_solver_within_tolerance(name):
    case = CASES[name]()
    g, o = _pair(case)
    g.iterations(300)
    o.iterations(300)
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert relerr(gs[k], os_[k]) < HYBRID_TOL, (k, relerr(gs[k], os_[k]))


def test_natural_cavity_64_two_thousand_iterations():
    # the plain small configuration: 64x64, Ra=1e4, 2000 outer iterations
    case = cases.natural_cavity(64, 64, Ra=1e4, T0=0.5)
    g, o = _pair(case)
    g.iterations(2000)
    o.iterations(2000)
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert relerr(gs[k], os_[k]) < HYBRID_TOL, (k, relerr(gs[k], os_[k]))
    ng = g.nusselt_x(2, 62)
    no = o.nusselt_x(2, 62)
    assert abs(ng[0] - no[0]) < 1e-10 and abs(ng[1] - no[1]) < 1e-10


@pytest.mark.parametrize("shape", Simple2D.SHAPES)
def test_every_launch_shape_keeps_parity(shape):
    case = cases.lid_driven_mixed(45, 29)
    g, o = _pair(case)
    for k in range(8):
        g.set_sweep_shape(k, *shape)
    g.iterations(60)
    o.iterations(60)
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert relerr(gs[k], os_[k]) < HYBRID_TOL, (k, relerr(gs[k], os_[k]))


def test_iteration_launch_count():
    if os.environ.get("IXB_SPLIT") == "1":
        pytest.skip("fused sweeps switched off")
    g = Simple2D.from_case(cases.lid_driven_mixed(45, 29))
    # plus the correction and the residual (the graph's do-while pressure
    # loop starts from the zero field: no p' reset kernel); the residual
    # rides on the T-x sweep when that sweep runs fused
    for k in range(8):
        g.set_sweep_shape(k, 1, 128)  # x-sweeps fused, y-sweeps two kernels
    assert g.iteration_launches() == 4 * 1 + 4 * 2 + 1
    for k in range(8):
        g.set_sweep_shape(k, 4, 64)  # y-sweeps fused, x-sweeps two kernels
    assert g.iteration_launches() == 4 * 2 + 4 * 1 + 2
    g.set_sweep_shape(1, 1, 256)
    assert g.iteration_launches() == 3 * 2 + 5 * 1 + 2
    g.set_sweep_shape(7, 1, 256)  # T-x fused as well
    assert g.iteration_launches() == 2 * 2 + 6 * 1 + 1


_SPLIT_CHILD = """
import os
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from ixchel2d_b200 import Simple2D, cases
from ixchel2d_b200 import _ffi as F
from oracle import oracle as O
from tests.conftest import relerr
STATE = ("u", "v", "p", "T", "u_ant", "v_ant", "T_ant")
case = cases.lid_driven_mixed(45, 29)
for solver, iters in ((F.SOLVER_EXACT, 40), (F.SOLVER_HYBRID, 200)):
    for shape in ((1, 128), (1, 256)):
        g = Simple2D.from_case(case, solver=solver)
        o = O.OracleCase(case, solver=solver)
        for k in range(8):
            g.set_sweep_shape(k, *shape)
        assert g.iteration_launches() == 18, g.iteration_launches()
        g.iterations(iters)
        o.iterations(iters)
        gs, os_ = g.download(), o.get_state()
        for k in STATE:
            if solver == F.SOLVER_EXACT:
                assert np.array_equal(gs[k], os_[k]), (k, shape)
            else:
                assert relerr(gs[k], os_[k]) < 1e-10, (k, shape, relerr(gs[k], os_[k]))
print("ok")
"""


def test_two_kernel_form_keeps_parity():
    # IXB_SPLIT=1 (read once per process) keeps every sweep at two kernels,
    # assembly and line solve: parity of that form for the one-line x shapes
    # that otherwise run fused, in a child process
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _SPLIT_CHILD, root], env={**os.environ, "IXB_SPLIT": "1"},
                       capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-2000:]


_STRIDED_CHILD = r"""
import sys
sys.path.insert(0, sys.argv[1])
import numpy as np
import torch
from ixchel2d_b200 import _ffi as F
from oracle import oracle as O
from tests.conftest import relerr
for n, nsys in ((5, 16), (48, 64), (300, 48), (700, 64), (1025, 36), (2048, 128), (2049, 16), (3000, 100),
                (4096, 512)):
    rng = np.random.default_rng(n + 3 * nsys)
    a = rng.uniform(-1, 0, (nsys, n)); c = rng.uniform(-1, 0, (nsys, n))
    b = np.abs(a) + np.abs(c) + rng.uniform(0.1, 1, (nsys, n)); d = rng.uniform(-1, 1, (nsys, n))
    ref = O.tridiagonal_batch(a, b, c, d)
    for tdt, fn, tol in ((torch.float64, F.lib.ixb_tridiag_f64, 1e-12), (torch.float32, F.lib.ixb_tridiag_f32, 2e-5)):
        A, B, Cc, D = (torch.tensor(np.ascontiguousarray(v.T), dtype=tdt, device="cuda") for v in (a, b, c, d))
        X = torch.full_like(D, float("nan"))
        st = fn(A.data_ptr(), B.data_ptr(), Cc.data_ptr(), D.data_ptr(), X.data_ptr(), n, nsys, 1, F.SOLVER_HYBRID,
                torch.cuda.current_stream().cuda_stream)
        assert st == F.OK, (n, nsys, st)
        torch.cuda.synchronize()
        e = relerr(X.cpu().numpy().astype(np.float64).T, ref)
        assert e < tol, (n, nsys, str(tdt), e)
        assert F.lib.ixb_tridiag_status() == F.OK, (n, nsys)
print("ok")
"""


@pytest.mark.parametrize("seg", ["64", "128"])
def test_strided_configurations_keep_parity(seg):
    # IXB_STRIDED_SEG (read once per process) forces one interleaved cluster
    # configuration for every size: 64-byte segments with 512-row CTAs, or
    # 128-byte segments with 256-row CTAs; every row is written (X starts as NaN)
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _STRIDED_CHILD, root], env={**os.environ, "IXB_STRIDED_SEG": seg},
                       capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-2000:]


def test_autotune_then_parity():
    case = cases.natural_cavity(40, 36, Ra=1e5)
    g, o = _pair(case)
    before = g.download()
    chosen = g.autotune(reps=2)
    after = g.download()
    for k in STATE:
        assert np.array_equal(before[k], after[k]), k  # state restored
    assert all((c[0], c[1]) in Simple2D.SHAPES for c in chosen.values())
    g.iterations(80)
    o.iterations(80)
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert relerr(gs[k], os_[k]) < HYBRID_TOL, k


def test_graph_and_host_driven_loops_agree(monkeypatch):
    case = cases.natural_cavity(20, 24, Ra=1e4)
    over = dict(conv_u=2e-3, conv_p=5e-3, conv_t=1e-3, iter_ecuaci_max=3, iter_simple_max=6,
                conv_paso=0.0, conv_resi=0.0)
    g1 = Simple2D.from_case(case, **over)
    monkeypatch.setenv("IXB_NO_GRAPH", "1")
    g2 = Simple2D.from_case(case, **over)
    r1 = g1.loop()
    r2 = g2.loop()
    for k in ("n_simple", "n_momen", "n_pres", "n_ener", "exit_code"):
        assert r1[k] == r2[k], k
    s1, s2 = g1.download(), g2.download()
    for k in STATE:
        assert np.array_equal(s1[k], s2[k]), k


def test_loop_exit_logic_matches_oracle():
    case = cases.natural_cavity(20, 24, Ra=1e4)
    over = dict(conv_u=2e-3, conv_p=5e-3, conv_t=1e-3, iter_ecuaci_max=3, iter_simple_max=6,
                conv_paso=0.0, conv_resi=0.0, solver=F.SOLVER_EXACT)
    g, o = _pair(case, **over)
    rg = g.loop()
    ro = o.loop()
    for k in ("n_simple", "n_momen", "n_pres", "n_ener", "exit_code"):
        assert rg[k] == ro[k], (k, rg[k], ro[k])
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert np.array_equal(gs[k], os_[k]), k


@pytest.mark.parametrize("n", [4, 7, 12])
def test_fixed_counts_through_the_unrolled_graph(n):
    # multiples of 4 run with four outer passes per WHILE body, other counts
    # in the plain graph: the same fields as n single calls, and the counts
    case = cases.natural_cavity(20, 16, Ra=1e5)
    a, b = _pair(case, solver=F.SOLVER_EXACT)[0], Simple2D.from_case(case, solver=F.SOLVER_EXACT)
    rep = a.iterations(n)
    for _ in range(n):
        b.iterations(1)
    assert rep["n_simple"] == n and rep["n_momen"] == n and rep["n_pres"] == n and rep["n_ener"] == n, rep
    sa, sb = a.download(), b.download()
    for k in STATE:
        assert np.array_equal(sa[k], sb[k]), k


def test_time_steps_with_roll():
    case = cases.natural_cavity(16, 16, Ra=1e4, dt=0.5, iter_simple_max=3)
    g, o = _pair(case, solver=F.SOLVER_EXACT)
    for _ in range(3):
        g.step()
        o.loop()
        o.roll()
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert np.array_equal(gs[k], os_[k]), k


def test_converged_exit_on_mass_residual():
    case = cases.natural_cavity(16, 16, Ra=1e3)
    over = dict(conv_paso=1e-6, conv_resi=1e-6, iter_simple_max=5000)
    g, o = _pair(case, **over)
    rg, ro = g.loop(), o.loop()
    assert rg["exit_code"] == 1 == ro["exit_code"]
    assert abs(rg["n_simple"] - ro["n_simple"]) <= 1
    assert rg["maxbo"] < 1e-6 and rg["residuo"] < 1e-6


def test_sources_immersed_block():
    # an immersed square through the source-term penalty of
    # definir_cuerpo (mod_front_inmersa.f90:121-125)
    case = cases.natural_cavity(24, 24, Ra=1e4)
    mi, nj = case.mi, case.nj
    fu = np.zeros((mi, nj + 1), order="F"); lu = np.zeros_like(fu)
    fv = np.zeros((mi + 1, nj), order="F"); lv = np.zeros_like(fv)
    fu[9:14, 9:14] = 10.0e50 * 10.0e-12; lu[9:14, 9:14] = -10.0e50
    fv[9:14, 9:14] = 10.0e50 * 10.0e-12; lv[9:14, 9:14] = -10.0e50
    case.sources = {0: (fu, lu), 1: (fv, lv)}
    g, o = _pair(case, solver=F.SOLVER_EXACT)
    g.iterations(30)
    o.iterations(30)
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert np.array_equal(gs[k], os_[k]), k


def test_sources_body_holding_temperature():
    # a solid block from ixb_body_sources: u, v and T penalty sources, T held
    # at 0.25 (definir_cuerpo's 'chime' form, mod_front_inmersa.f90:135-177)
    case = cases.natural_cavity(24, 24, Ra=1e4)
    cases.add_body(case, F.BODY_BOX, [0.4, 0.6, 0.3, 0.55], F.BODY_VEL | F.BODY_TEMP, 0.25)
    assert set(case.sources) == {0, 1, 2}
    g, o = _pair(case, solver=F.SOLVER_EXACT)
    g.iterations(30)
    o.iterations(30)
    gs, os_ = g.download(), o.get_state()
    for k in STATE:
        assert np.array_equal(gs[k], os_[k]), k
    body = case.sources[2][1] != 0
    assert body.sum() > 4
    assert np.allclose(gs["T"][body], 0.25, rtol=0, atol=1e-12)
    # the reference's pair (1e40, -1e51) holds u and v at 1e-11
    ub = gs["u"][case.sources[0][1] != 0]
    assert np.allclose(ub, 1e-11, rtol=1e-9, atol=0)


def test_nusselt_matches_oracle():
    case = cases.natural_cavity(32, 32, Ra=1e4)
    g, o = _pair(case)
    g.iterations(200)
    o.iterations(200)
    for fn, rng_ in (("nusselt_x", (2, 30)), ("nusselt_y", (3, 27))):
        a = getattr(g, fn)(*rng_)
        b = getattr(o, fn)(*rng_)
        assert abs(a[0] - b[0]) < 1e-9 and abs(a[1] - b[1]) < 1e-9, fn


def test_nonfinite_norm_is_reported():
    case = cases.natural_cavity(16, 16)
    case.state["T"][5, 5] = np.nan
    g = Simple2D.from_case(case)
    with pytest.raises(IxbError) as ei:
        g.iterations(3)
    assert ei.value.status == F.ENONFINITE


def test_uncovered_boundary_table_is_rejected():
    case = cases.natural_cavity(16, 16)
    g = Simple2D(16, 16)
    # side a of T covers only lines 2..8 (a 'desc' segment after it)
    sides = cases.bc_table((case.xp, case.yp), {0: [(0.5, F.BC_DIRI, 1.0), (2.0, F.BC_OTHER, 0.0)],
                                                1: [(9.0, F.BC_NEUM, 0.0)], 2: [(9.0, F.BC_DIRI, 0.0)],
                                                3: [(9.0, F.BC_NEUM, 0.0)]})
    with pytest.raises(IxbError) as ei:
        g.set_bc(2, sides)
    assert ei.value.status == F.EBC


def test_simple_before_setup_is_refused():
    g = Simple2D(16, 16)
    with pytest.raises(IxbError) as ei:
        g.iterations(1)
    assert ei.value.status == F.ESTATE


# ---------------------------------------------------------------------------
# batched tridiagonal entry points (device pointers via torch)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("n,nsys", [(5, 3), (65, 40), (702, 33), (4096, 9), (4096, 400), (2050, 333),
                                    (300, 48), (700, 64), (1025, 36), (3000, 100), (4096, 512)])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("solver", [F.SOLVER_EXACT, F.SOLVER_HYBRID])
def test_tridiag_batch(layout, n, nsys, dtype, solver):
    import torch
    rng = np.random.default_rng(n * 7 + nsys)
    a = rng.uniform(-1, 0, (nsys, n)); c = rng.uniform(-1, 0, (nsys, n))
    b = np.abs(a) + np.abs(c) + rng.uniform(0.1, 1, (nsys, n)); d = rng.uniform(-1, 1, (nsys, n))
    ref = O.tridiagonal_batch(a, b, c, d)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    conv = (lambda x: torch.tensor(x, dtype=tdt, device="cuda").contiguous()) if layout == 0 else \
        (lambda x: torch.tensor(np.ascontiguousarray(x.T), dtype=tdt, device="cuda"))
    A, B, Cc, D = map(conv, (a, b, c, d))
    X = torch.empty_like(D)
    fn = F.lib.ixb_tridiag_f64 if dtype == "f64" else F.lib.ixb_tridiag_f32
    st = fn(A.data_ptr(), B.data_ptr(), Cc.data_ptr(), D.data_ptr(), X.data_ptr(), n, nsys, layout, solver,
            torch.cuda.current_stream().cuda_stream)
    assert st == F.OK
    torch.cuda.synchronize()
    x = X.cpu().numpy().astype(np.float64)
    if layout == 1:
        x = x.T
    if dtype == "f64" and solver == F.SOLVER_EXACT:
        assert np.array_equal(x, ref)
    else:
        tol = 1e-12 if dtype == "f64" else 2e-5
        assert relerr(x, ref) < tol, relerr(x, ref)
    assert F.lib.ixb_tridiag_status() == F.OK  # no bounded copy wait expired


def test_u_buoyancy_keeps_parity():
    # the u residual reads T (Ri != 0: a nonzero buoyancy term in the u rows
    # and the residual); exact mode stays bit-identical to the oracle
    for ri in (0.0, 0.3):
        case = cases.lid_driven_mixed(37, 23, Re=100.0, Ri=1.0)
        case.params["Ri"] = ri
        g, o = _pair(case, solver=F.SOLVER_EXACT)
        rg = g.iterations(30)
        ro = o.iterations(30)
        gs, os_ = g.download(), o.get_state()
        for k in STATE:
            assert np.array_equal(gs[k], os_[k]), (ri, k, relerr(gs[k], os_[k]))
        assert abs(rg["residuo"] - ro["residuo"]) <= 1e-12 * abs(ro["residuo"]), ri
