"""The ixchel2d_gpu case driver (PROGRAM IXCHEL2D, source/main.f90, on the
C ABI): parametros.dat / mesh / boundary files in, Nusselt and out_* files
out, in the reference's formats.

CPU tests run the driver with --check (every input read, no GPU call).  GPU
tests run a 16x12 natural-convection case for 2000 time steps and compare
every file it writes with the oracle's run of the same steps: bit-identical
text with --solver exact; |dNu| < 1e-6 with --prec refined.
"""
import numpy as np
import pytest

from ixchel2d_b200 import cases
from ixchel2d_b200 import casefiles as CF
from oracle import oracle as O

MI, NJ = 16, 12
PRM = dict(adimen="natural", Ra=1e4, Pr=0.71, Ri_1=0.0, dt=0.5, paq_itera=1000, itermax=2000, rel_pres=0.3,
           rel_vel=0.7, rel_ener=0.9, conv_u=1e-6, conv_t=1e-6, conv_p=1e-6, conv_resi=1e-6, conv_paso=1e-6,
           iter_ecuaci_max=5, iter_simple_max=10, flujo_ini="nulo", tempe_ini="archivo", postprocesar=True)


def _case_dir(path, **over):
    prm = dict(PRM)
    make_folder = over.pop("make_folder", True)
    prm.update(over)
    mesh = cases.staggered_mesh(MI, NJ)
    state = cases.zero_state(MI, NJ, 0.5)
    names = CF.write_case_dir(path, MI, NJ, mesh, CF.natural_cavity_segments(), prm, state,
                              make_folder=make_folder)
    return names, mesh, state


def _check(path, *args):
    r = CF.run_driver(path, "--check", *args, timeout=120)
    kv = {}
    for line in r.stdout.splitlines():
        if "=" in line and not line.startswith(" "):
            k, v = line.split("=", 1)
            kv[k] = v
    return r, kv


def test_d23_15_text_matches_the_library(tmp_path):
    """The Python D23.15 formatter the GPU tests compare with writes what
    the library's file writer writes."""
    rng = np.random.default_rng(5)
    vals = np.concatenate([rng.standard_normal(40) * 10.0 ** rng.integers(-120, 120, 40),
                           [0.0, 1.0, -1.0, 0.1, 9.9999999999999995e-7, 123456.789, 1e-300, -2.5e100]])
    mi, nj = 2, 2
    z = [np.zeros(s, order="F") for s in ((mi + 1, nj), (mi + 1, nj + 1), (mi + 1, nj + 1))]
    mesh = (np.arange(mi, dtype=float), np.arange(nj, dtype=float), np.arange(mi + 1, dtype=float),
            np.arange(nj + 1, dtype=float))
    for start in range(0, len(vals), mi * (nj + 1)):
        chunk = vals[start:start + mi * (nj + 1)]
        u = np.zeros((mi, nj + 1), order="F")
        u.T.flat[:len(chunk)] = chunk
        names = tuple(str(tmp_path / n) for n in ("u.dat", "v.dat", "p.dat"))
        CF.write_state_files(names, mi, nj, mesh, {"u": u, "v": z[0], "T": z[1], "p": z[2]}, 1, 1, 0, 1.0)
        lines = (tmp_path / "u.dat").read_text().splitlines()[1:]
        for line, x in zip(lines, u.T.ravel()):
            assert line[46:69] == CF.fmt_d23_15(x), (line, x)


def test_check_reads_the_case(tmp_path):
    names, mesh, _ = _case_dir(tmp_path)
    r, kv = _check(tmp_path)
    assert r.returncode == 0, r.stderr
    assert (int(kv["mi"]), int(kv["nj"])) == (MI, NJ)  # inferred from the record counts
    nd = cases.nondim("natural", 1e4, 0.71, 0.0)
    for k in ("gamma_momen", "gamma_energ", "Ri", "Riy"):
        assert float(kv[k]) == nd[k], k
    assert kv["Rec"] == "00100" == names["rec"]
    assert kv["nusselt_file"] == names["nusselt"] == "nuss_sim_n00012m00016_R00100.dat"
    assert kv["folder"] == names["folder"]
    assert (int(kv["placa_min"]), int(kv["placa_max"])) == (names["i0"], names["i1"])
    assert int(kv["postprocesar"]) == 1 and kv["flujo_ini"] == "nulo" and kv["tempe_ini"] == "archivo"
    info = (tmp_path / names["folder"] / "info_entrada.out").read_text().splitlines()
    assert len(info) == 21 and "numero de Rayleigh" in info[0] and "10000.000000000000" in info[0]


def test_fortran_spellings_of_parametros(tmp_path):
    """List-directed input as gfortran reads it: D exponents, unquoted
    strings truncated to the variable's length, T/F logicals, blank records
    and trailing comments; 'mixta' mode with Re = ceiling(Ra)."""
    names, _, _ = _case_dir(tmp_path)
    lines = [
        "mixta          ! adimen",
        "150.3d0        ! Re",
        "",
        "0.71D+00, ignored",
        "2.5            ! Ri",
        "1.0d-2",
        "10",
        "20",
        "0.3", "0.7", "0.9",
        "1.d-6", "1.0E-6", "1e-6", "1e-6", "1e-6",
        "5", "10",
        "n12m16u.dat", "n12m16v.dat", "n12m16p.dat",
        "archivo_largo   ! character(len=8) keeps 'archivo_'",
        "alta",
        "T",
    ]
    (tmp_path / "parametros.dat").write_text("\n".join(lines) + "\n")
    rec = CF.reynolds_tag("mixta", 150.3)
    assert rec == "00151"
    (tmp_path / f"n00012m00016R{rec}").mkdir()
    r, kv = _check(tmp_path)
    assert r.returncode == 0, r.stderr
    assert kv["adimen"] == "mixta" and kv["Rec"] == rec
    assert float(kv["gamma_momen"]) == 1.0 / 150.3
    assert float(kv["gamma_energ"]) == 1.0 / (150.3 * 0.71)
    assert float(kv["Riy"]) == 2.5 and float(kv["Ri"]) == 0.0
    assert float(kv["dt"]) == 1.0e-2 and float(kv["conv_u"]) == 1e-6
    assert kv["flujo_ini"] == "archivo_" and kv["tempe_ini"] == "alta"
    assert int(kv["postprocesar"]) == 1 and int(kv["paq_itera"]) == 10 and int(kv["itermax"]) == 20


def test_missing_output_folder_is_an_error(tmp_path):
    names, _, _ = _case_dir(tmp_path, make_folder=False)
    r, _ = _check(tmp_path)
    assert r.returncode == 2 and names["folder"] in r.stderr
    r, kv = _check(tmp_path, "--mkdir")
    assert r.returncode == 0 and (tmp_path / names["folder"] / "info_entrada.out").exists()


@pytest.mark.parametrize("bad,needle", [
    ({"adimen": "forzada"}, "adimen"),
    ({"paq_itera": 0}, "paq_itera"),
])
def test_bad_parametros_are_errors(tmp_path, bad, needle):
    _case_dir(tmp_path, **bad)
    r, _ = _check(tmp_path)
    assert r.returncode == 2 and needle in r.stderr


def test_truncated_parametros_is_an_error(tmp_path):
    _case_dir(tmp_path)
    lines = (tmp_path / "parametros.dat").read_text().splitlines()
    (tmp_path / "parametros.dat").write_text("\n".join(lines[:10]) + "\n")
    r, _ = _check(tmp_path)
    assert r.returncode == 2 and "record 11" in r.stderr and "conv_u" in r.stderr


def test_wrong_grid_size_is_an_error(tmp_path):
    _case_dir(tmp_path)
    r, _ = _check(tmp_path, "--mi", str(MI - 1), "--nj", str(NJ))
    assert r.returncode == 2 and "staggered mesh" in r.stderr
    r, kv = _check(tmp_path, "--mi", str(MI), "--nj", str(NJ))
    assert r.returncode == 0 and int(kv["mi"]) == MI


# ---------------------------------------------------------------------------
# GPU: the run against the oracle's run of the same 2000 time steps
# ---------------------------------------------------------------------------

@pytest.fixture(scope="module")
def oracle_run():
    """The oracle stepping the case as main.f90 does: Nusselt records after
    1000 and 2000 steps, the final state."""
    segs = CF.natural_cavity_segments()
    xu, yv, xp, yp = cases.staggered_mesh(MI, NJ)
    bc = {0: cases.bc_table((xu, yp), segs[0]), 1: cases.bc_table((xp, yv), segs[1]),
          2: cases.bc_table((xp, yp), segs[2])}
    prm = cases.default_params(**cases.nondim("natural", PRM["Ra"], PRM["Pr"], 0.0))
    for k in ("dt", "rel_pres", "rel_vel", "rel_ener", "conv_u", "conv_t", "conv_p", "conv_resi", "conv_paso",
              "iter_ecuaci_max", "iter_simple_max"):
        prm[k] = PRM[k]
    prm["solver"] = 1
    case = cases.Case(MI, NJ, xu, yv, xp, yp, prm, bc, cases.zero_state(MI, NJ, 0.5))
    o = O.OracleCase(case)
    i0 = 1
    i1 = MI - 1 if (MI - 1 - i0) % 2 == 0 else MI - 2
    rows = []
    for itera in range(1, PRM["itermax"] + 1):
        o.loop()
        o.roll()
        if itera % 1000 == 0:
            nu0, nu1 = o.nusselt_y(i0, i1)
            T = o.get_state()["T"]
            ic, jc = (i0 + i1) // 2, NJ // 2 + 1
            t_med = (T[ic - 1, jc - 1] + T[ic, jc - 1]) / 2.0
            rows.append((itera * PRM["dt"], nu0, -nu1, t_med, 0.0, 0.0))
    st = o.get_state()
    o.close()
    return rows, st, (xu, yv, xp, yp)


def _need_gpu(has_gpu):
    if not has_gpu:
        pytest.skip("no CUDA device")


@pytest.mark.gpu
def test_driver_exact_run_matches_oracle(tmp_path, has_gpu, oracle_run):
    _need_gpu(has_gpu)
    rows, st, (xu, yv, xp, yp) = oracle_run
    names, _, _ = _case_dir(tmp_path)
    r = CF.run_driver(tmp_path, "--solver", "exact", timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout[-2000:]
    assert "itera_total=        2000" in r.stdout and r.stdout.count("ITERACION:") == 4

    # Nusselt records: identical text (form26)
    got = (tmp_path / names["nusselt"]).read_text().splitlines()
    want = ["".join(CF.fmt_d23_15(x) for x in row) for row in rows]
    assert got == want

    # out_*.dat: the final fields through D23.15, header (placa_min, placa_max, itera_total, ao)
    out = CF.read_out_files(tuple(tmp_path / names[k] for k in ("out_u", "out_v", "out_p")), MI, NJ)
    assert (out["i0"], out["i1"], out["iter"], out["ao"]) == (names["i0"], names["i1"], 2000, 1.0)
    for k in ("u", "v", "T", "p"):
        want_k = cases.d23_15(st[k].ravel(order="F")).reshape(st[k].shape, order="F")
        assert np.array_equal(out[k], want_k), k

    # out_*.bin: the final fields exactly
    bp = np.frombuffer((tmp_path / names["bin_p"]).read_bytes(), dtype="<f8").reshape(NJ + 1, MI + 1, 2)
    assert np.array_equal(bp[..., 0], st["T"].T) and np.array_equal(bp[..., 1], st["p"].T)
    bu = np.frombuffer((tmp_path / names["bin_u"]).read_bytes(), dtype="<f8").reshape(NJ + 1, MI, 3)
    assert np.array_equal(bu[..., 2], st["u"].T) and np.array_equal(bu[0, :, 0], xu)
    bv = np.frombuffer((tmp_path / names["bin_v"]).read_bytes(), dtype="<f8").reshape(NJ, MI + 1, 3)
    assert np.array_equal(bv[..., 2], st["v"].T) and np.array_equal(bv[:, 0, 1], yv)

    # the VTK file of the second package: itera_total 2000 with paq_itera 1000 -> t_00020.vtk
    vtk = (tmp_path / names["folder"] / "t_00020.vtk").read_bytes()
    npts = (MI + 1) * (NJ + 1)
    head = (b"# vtk DataFile Version 2.3\n3D Mesh\nBINARY\nDATASET STRUCTURED_GRID\n"
            + b"DIMENSIONS " + b"%12d%12d%12d" % (MI + 1, NJ + 1, 1) + b"\nPOINTS " + b"%12d" % npts + b" float\n")
    assert vtk.startswith(head)
    k = len(head) + 12 * npts
    tail = b"\nPOINT_DATA " + b"%12d" % npts + b"SCALARS PRESS float\nLOOKUP_TABLE default\n"
    assert vtk[k:k + len(tail)] == tail
    k += len(tail) + 4 * npts
    tail = b"\nSCALARS TEMPER float\nLOOKUP_TABLE default\n"
    assert vtk[k:k + len(tail)] == tail
    k += len(tail)
    T32 = np.frombuffer(vtk[k:k + 4 * npts], dtype=">f4")
    assert np.array_equal(T32, st["T"].T.astype(np.float32).ravel())
    assert len(vtk) == k + 4 * npts + len(b"\nVECTORS VELOCITY float\n") + 12 * npts
    assert (tmp_path / names["folder"] / "t_00010.vtk").exists()


@pytest.mark.gpu
def test_driver_refined_run_keeps_nusselt(tmp_path, has_gpu, oracle_run):
    """FP32 line solves refined to binary64: the Nusselt records within 1e-6
    of the binary64 oracle."""
    _need_gpu(has_gpu)
    rows, _, _ = oracle_run
    names, _, _ = _case_dir(tmp_path, postprocesar=False)
    r = CF.run_driver(tmp_path, "--prec", "refined", "--quiet", timeout=600)
    assert r.returncode == 0, r.stderr
    got = CF.read_nusselt(tmp_path / names["nusselt"])
    want = np.array(rows)
    assert got.shape == want.shape
    assert np.max(np.abs(got[:, 1:3] - want[:, 1:3])) < 1e-6
    assert np.max(np.abs(got[:, 3] - want[:, 3])) < 1e-6
    assert not (tmp_path / names["out_u"]).exists()


def test_reynolds_tag_overflows_like_the_reference(tmp_path):
    """entero_caracter writes each of its five digits with I1, so a ten-
    thousands digit above 9 prints '*' (Re = ceiling(sqrt(1e12)) = 1e6)."""
    assert CF.entero_caracter(1_000_000) == "*0000"
    assert CF.entero_caracter(99_999) == "99999"
    rec = CF.reynolds_tag("natural", 1e12)
    assert rec == "*0000"
    _case_dir(tmp_path, Ra=1e12, make_folder=False)
    r, kv = _check(tmp_path, "--mkdir")
    assert r.returncode == 0, r.stderr
    assert kv["Rec"] == rec and kv["folder"] == f"n00012m00016R{rec}"
    assert kv["nusselt_file"] == f"nuss_sim_n00012m00016_R{rec}.dat"
