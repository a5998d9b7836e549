"""Case folders in the reference's file formats, and the ``ixchel2d_gpu``
driver that runs them.

A case folder is what ``PROGRAM IXCHEL2D`` (source/main.f90) reads from its
working directory:

* ``parametros.dat``: 23 list-directed records (main.f90:164-189);
* the three mesh/state files it names (header ``i_0 i_1 iter a``, then
  D23.15 records; mod_malla.f90:137-162);
* ``cond_frontera{u,v,t}.dat``: per side ``variable lado ndivis``, then
  ``ndivis`` records ``x0 x1 tipo valor`` (mod_cond_frontera.f90:109-135);
* the output folder ``n<nj>m<mi>R<Re>/`` that must exist before the run.

:func:`write_case_dir` writes one, :func:`run_driver` runs the driver on it
and :func:`read_nusselt` / :func:`read_out_files` read what it writes.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from pathlib import Path

import numpy as np

from ._ffi import BC_DIRI, BC_NEUM, check, dptr, lib

PKG = Path(__file__).resolve().parent
DRIVER = PKG / "ixchel2d_gpu"

SIDES = "abcd"
VARS = ("u", "v", "t")
_TIPO = {BC_DIRI: "diri", BC_NEUM: "neum"}


def entero_caracter(e: int) -> str:
    """entero_caracter (mod_postproceso.f90:375-401): five I1 digits."""
    out = []
    for d in (e // 10000, (e % 10000) // 1000, (e % 1000) // 100, (e % 100) // 10, e % 10):
        out.append(str(d) if 0 <= d <= 9 else "*")
    return "".join(out)


def reynolds_tag(adimen: str, Ra: float) -> str:
    """The ``Rec`` string of main.f90:225-241."""
    return entero_caracter(math.ceil(math.sqrt(Ra)) if adimen == "natural" else math.ceil(Ra))


def case_names(mi: int, nj: int, adimen: str, Ra: float) -> dict:
    """File and folder names the reference derives from mi, nj and Re."""
    rec = reynolds_tag(adimen, Ra)
    tag = f"n{entero_caracter(nj)}m{entero_caracter(mi)}_R{rec}"
    return {"folder": f"n{entero_caracter(nj)}m{entero_caracter(mi)}R{rec}", "nusselt": f"nuss_sim_{tag}.dat",
            "out_u": f"out_{tag}u.dat", "out_v": f"out_{tag}v.dat", "out_p": f"out_{tag}p.dat",
            "bin_u": f"out_{tag}u.bin", "bin_v": f"out_{tag}v.bin", "bin_p": f"out_{tag}p.bin", "rec": rec}


def fmt_d23_15(x: float) -> str:
    """x as Fortran's D23.15 edit writes it."""
    x = float(x)
    if x == 0.0:
        s = "0.000000000000000D+00"
    else:
        mant, ex = f"{abs(x):.14E}".split("E")
        e = int(ex) + 1
        exps = f"D{'-' if e < 0 else '+'}{abs(e):02d}" if abs(e) <= 99 else f"{'-' if e < 0 else '+'}{abs(e):03d}"
        s = ("-" if x < 0 else "") + "0." + mant.replace(".", "") + exps
    return s.rjust(23)


def _q(s: str) -> str:
    return "'" + s.replace("'", "''") + "'"


def parametros_text(p: dict) -> str:
    """parametros.dat with one record per line and the reference's comments."""
    logical = ".true." if p.get("postprocesar", False) else ".false."
    rows = [
        (_q(p.get("adimen", "natural")), "adimen: natural | mixta"),
        (repr(float(p["Ra"])), "Rayleigh (natural) or Reynolds (mixta)"),
        (repr(float(p.get("Pr", 0.71))), "Prandtl"),
        (repr(float(p.get("Ri_1", 0.0))), "Richardson"),
        (repr(float(p["dt"])), "time step"),
        (str(int(p["paq_itera"])), "time steps per package"),
        (str(int(p["itermax"])), "time steps of the run"),
        (repr(float(p.get("rel_pres", 0.3))), "pressure relaxation"),
        (repr(float(p.get("rel_vel", 0.7))), "velocity relaxation"),
        (repr(float(p.get("rel_ener", 0.9))), "temperature relaxation"),
        (repr(float(p["conv_u"])), "velocity convergence"),
        (repr(float(p["conv_t"])), "temperature convergence"),
        (repr(float(p["conv_p"])), "pressure convergence"),
        (repr(float(p["conv_resi"])), "residual convergence"),
        (repr(float(p["conv_paso"])), "time-step convergence"),
        (str(int(p["iter_ecuaci_max"])), "inner iterations per equation"),
        (str(int(p["iter_simple_max"])), "SIMPLE iterations per time step"),
        (_q(p["entrada_u"]), "u mesh/state file"),
        (_q(p["entrada_v"]), "v mesh/state file"),
        (_q(p["entrada_tp"]), "T/p mesh/state file"),
        (_q(p.get("flujo_ini", "nulo")), "initial flow: nulo | archivo"),
        (_q(p.get("tempe_ini", "archivo")), "initial temperature: baja | alta | archivo"),
        (logical, "write out_* and VTK files after every package"),
    ]
    return "".join(f"{v:<22} ! {c}\n" for v, c in rows)


def bc_file_text(var: str, sides: dict[int, list[tuple[float, int, float]]]) -> str:
    """cond_frontera<var>.dat: segments are (x1, type, value) per side in file
    order, as the located tables of cases.bc_table take them."""
    out = []
    for s in range(4):
        segs = sides.get(s, [])
        out.append(f"{_q(var)} {_q(SIDES[s])} {len(segs)}\n")
        x0 = 0.0
        for x1, ty, val in segs:
            out.append(f"{x0!r} {float(x1)!r} {_q(_TIPO.get(ty, 'desc'))} {float(val)!r}\n")
            x0 = float(x1)
    return "".join(out)


def write_state_files(names: tuple[str, str, str], mi: int, nj: int, mesh, state: dict, i0: int, i1: int,
                      iteration: int, ao: float) -> None:
    """The three D23.15 mesh/state files (ixb_write_state_files)."""
    xu, yv, xp, yp = (np.ascontiguousarray(a, dtype=np.float64) for a in mesh)
    u, v, T, p = (np.asfortranarray(state[k], dtype=np.float64) for k in ("u", "v", "T", "p"))
    check(lib.ixb_write_state_files(*(n.encode() for n in names), mi, nj, *map(dptr, (xu, yv, xp, yp, u, v, T, p)),
                                    int(i0), int(i1), int(iteration), float(ao)), "ixb_write_state_files")


def read_out_files(names: tuple[str, str, str], mi: int, nj: int) -> dict:
    """Reads three mesh/state files back: mesh, fields and the header."""
    xu, yv, xp, yp = np.zeros(mi), np.zeros(nj), np.zeros(mi + 1), np.zeros(nj + 1)
    u = np.zeros((mi, nj + 1), order="F")
    v = np.zeros((mi + 1, nj), order="F")
    T = np.zeros((mi + 1, nj + 1), order="F")
    p = np.zeros((mi + 1, nj + 1), order="F")
    i0, i1, it, a = C.c_int(), C.c_int(), C.c_int(), C.c_double()
    check(lib.ixb_read_state_files(*(str(n).encode() for n in names), mi, nj,
                                   *map(dptr, (xu, yv, xp, yp, u, v, T, p)), C.byref(i0), C.byref(i1), C.byref(it),
                                   C.byref(a)), "ixb_read_state_files")
    return {"xu": xu, "yv": yv, "xp": xp, "yp": yp, "u": u, "v": v, "T": T, "p": p, "i0": i0.value,
            "i1": i1.value, "iter": it.value, "ao": a.value}


def write_case_dir(path, mi: int, nj: int, mesh, bc_segments: dict[int, dict[int, list]], parametros: dict,
                   state: dict, i0: int = 1, i1: int | None = None, iteration: int = 0, ao: float = 1.0,
                   make_folder: bool = True) -> dict:
    """Writes a complete case folder; returns case_names(...) for it.

    bc_segments: var (0 u, 1 v, 2 T) -> side -> [(x1, type, value), ...].
    parametros: the records of parametros.dat by name (file names default to
    n<nj>m<mi>{u,v,p}.dat).  i0, i1: the header's plate range, used by the
    Nusselt integral (default 1 .. the last odd index that fits)."""
    path = Path(path)
    path.mkdir(parents=True, exist_ok=True)
    prm = dict(parametros)
    base = f"n{nj}m{mi}"
    prm.setdefault("entrada_u", base + "u.dat")
    prm.setdefault("entrada_v", base + "v.dat")
    prm.setdefault("entrada_tp", base + "p.dat")
    if i1 is None:
        i1 = mi - 1 if (mi - 1 - i0) % 2 == 0 else mi - 2
    (path / "parametros.dat").write_text(parametros_text(prm))
    for var, name in enumerate(VARS):
        (path / f"cond_frontera{name}.dat").write_text(bc_file_text(name, bc_segments.get(var, {})))
    write_state_files(tuple(str(path / prm[k]) for k in ("entrada_u", "entrada_v", "entrada_tp")), mi, nj, mesh,
                      state, i0, i1, iteration, ao)
    names = case_names(mi, nj, prm.get("adimen", "natural"), float(prm["Ra"]))
    if make_folder:
        (path / names["folder"]).mkdir(exist_ok=True)
    names.update(i0=i0, i1=i1)
    return names


def natural_cavity_segments() -> dict:
    """Boundary segments of the differentially heated cavity: no-slip walls,
    T = 1 on side a (x = 0), T = 0 on side c, adiabatic sides b and d."""
    z = [(1e30, BC_DIRI, 0.0)]
    return {0: {s: z for s in range(4)}, 1: {s: z for s in range(4)},
            2: {0: [(1e30, BC_DIRI, 1.0)], 1: [(1e30, BC_NEUM, 0.0)], 2: [(1e30, BC_DIRI, 0.0)],
                3: [(1e30, BC_NEUM, 0.0)]}}


def driver_path() -> Path:
    """The built driver; builds it (and libixb.so) when missing."""
    if not DRIVER.exists():
        from .build import build
        build()
    return DRIVER


def run_driver(case_dir, *args: str, timeout: float = 600.0, env: dict | None = None) -> subprocess.CompletedProcess:
    """Runs ixchel2d_gpu on a case folder; returns the finished process."""
    e = dict(os.environ)
    if env:
        e.update(env)
    return subprocess.run([str(driver_path()), str(case_dir), *args], capture_output=True, text=True,
                          timeout=timeout, env=e)


def read_nusselt(path) -> np.ndarray:
    """nuss_sim_*.dat records (time, Nu0, -Nu1, T_med, T_int, S_int) as rows."""
    rows = []
    for line in Path(path).read_text().splitlines():
        if line.strip():
            rows.append([float(t.replace("D", "E")) for t in line.split()])
    return np.array(rows)
