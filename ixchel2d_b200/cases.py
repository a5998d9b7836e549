"""Synthetic Ixchel2D cases: staggered meshes, boundary tables, parameters
and initial states, built the way the reference's input files describe them.

* Meshes follow ``malla/malla_irr.f90``: u-nodes ``xu`` / v-nodes ``yv`` on
  the domain, p-nodes ``xp``/``yp`` at their midpoints plus one extrapolated
  node half a cell outside each wall (:97-106, :148-157).  ``tanh`` is a
  two-sided tanh wall clustering of the u/v nodes (malla_irr.f90 has only
  ``unif``/``tubo``/``cent``); ``tubo`` and ``cent`` restate the reference.
* Coordinates pass through the ``D23.15`` text format of the mesh files
  (mod_malla.f90:21, read at :137-162), i.e. 15 significant digits, so a
  case equals what the reference would read back from its own files.
* Boundary tables are one segment per side located by the rule of
  ``lectura_cond_frontera`` (mod_cond_frontera.f90:114-238).
* Parameters follow the non-dimensionalisation of main.f90:221-244.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from ._types import BC_DIRI, BC_NEUM, BCSide


def d23_15(x: np.ndarray) -> np.ndarray:
    """Round to the 15 significant digits of Fortran's D23.15 edit descriptor."""
    return np.array([float(f"{v:.14E}") for v in np.asarray(x, dtype=np.float64)], dtype=np.float64)


def _staggered(nodes: np.ndarray) -> np.ndarray:
    """p-node coordinates from u-node (or v-node) coordinates, malla_irr.f90:101-106."""
    n = nodes.size
    p = np.empty(n + 1)
    p[0] = (3.0 * nodes[0] - nodes[1]) / 2.0
    p[1:n] = (nodes[1:] + nodes[:-1]) / 2.0
    p[n] = (3.0 * nodes[n - 1] - nodes[n - 2]) / 2.0
    return p


def axis_nodes(kind: str, n: int, length: float = 1.0, param: float = 1.2, centre: float = 0.5) -> np.ndarray:
    """u- (or v-) node coordinates of one axis.

    unif: length*(i-1)/(n-1) (malla_irr.f90:97-100)
    tubo: erf wall clustering, ky=10, my=0.8 (malla_irr.f90:81-89)
    cent: sinh clustering around `centre`, tau=`param` (malla_irr.f90:54-64)
    tanh: length*(1+tanh(param*(2s-1))/tanh(param))/2, s=(i-1)/(n-1)
    """
    s = np.arange(n, dtype=np.float64) / float(n - 1)
    if kind == "unif":
        return length * 1.0 * s
    if kind == "tubo":
        ky, my = 10.0, 0.8
        erf = np.vectorize(math.erf)
        return length * 1.0 * (0.5 + my * (s - 0.5) + 0.5 * (1 - my) * erf(ky * (s - 0.5)) / math.erf(0.5 * ky))
    if kind == "cent":
        tau = param
        b = 1.0 / (2.0 * tau) * math.log((1.0 + (math.exp(tau) - 1.0) * (centre / length)) /
                                         (1.0 + (math.exp(-tau) - 1.0) * (centre / length)))
        return centre * (1.0 + np.sinh(tau * (s - b)) / math.sinh(tau * b))
    if kind == "tanh":
        return length * (1.0 + np.tanh(param * (2.0 * s - 1.0)) / math.tanh(param)) / 2.0
    raise ValueError(kind)


def staggered_mesh(mi: int, nj: int, xkind="unif", ykind="unif", ao=1.0, bo=1.0, xparam=1.2, yparam=1.2):
    xu = axis_nodes(xkind, mi, ao, xparam)
    yv = axis_nodes(ykind, nj, bo, yparam)
    xp = _staggered(xu)
    yp = _staggered(yv)
    return d23_15(xu), d23_15(yv), d23_15(xp), d23_15(yp)


def locate(coord: np.ndarray, x1s, size: int) -> list[int]:
    """Segment index list of one side, the rule of lectura_cond_frontera
    (source/mod_cond_frontera.f90:125-149): the first segment starts at node 2,
    segment k ends before the first node whose coordinate exceeds its x1
    (size+1 when none does), and the last segment ends at node size-1."""
    idx = [2]
    for x1 in x1s:
        kk = 1
        while kk <= size and not (coord[kk - 1] > x1):
            kk += 1
        idx.append(kk)
    idx[len(x1s)] = size - 1
    return idx


def bc_side(side: int, segments: list[tuple[float, int, float]], xx: np.ndarray, yy: np.ndarray) -> BCSide:
    """One side of a boundary table: segments are (x1, type, value) in file
    order; sides a and c (0, 2) run along the y-coordinates, b and d (1, 3)
    along x.  The same table ixb_bc_locate builds, computed here so that a
    case can be built without mapping the library."""
    if not 0 <= side <= 3 or len(segments) > 15:
        raise ValueError("side must be 0..3 and a side holds at most 15 segments")
    coord = np.asarray(yy if side in (0, 2) else xx, dtype=np.float64)
    out = BCSide()
    out.side = side
    out.ndivis = len(segments)
    for k, (_, ty, va) in enumerate(segments):
        out.type[k] = int(ty)
        out.value[k] = float(va)
    for k, ix in enumerate(locate(coord, [float(s[0]) for s in segments], coord.size)):
        out.index[k] = ix
    return out


def bc_table(var_nodes: tuple[np.ndarray, np.ndarray], sides: dict[int, list[tuple[float, int, float]]]):
    xx, yy = var_nodes
    return [bc_side(s, sides.get(s, []), xx, yy) for s in range(4)]


def side_dict(b: BCSide) -> dict:
    nd = b.ndivis
    return {"side": b.side, "ndivis": nd, "type": list(b.type[:nd]), "value": list(b.value[:nd]),
            "index": list(b.index[:nd + 1])}


@dataclass
class Case:
    """Everything the SIMPLE hot path consumes, in the reference's shapes."""
    mi: int
    nj: int
    xu: np.ndarray
    yv: np.ndarray
    xp: np.ndarray
    yp: np.ndarray
    params: dict
    bc: dict                      # var -> list of 4 BCSide
    state: dict                   # u v p T u_ant v_ant T_ant (Fortran-ordered arrays)
    sources: dict = field(default_factory=dict)  # var -> (fcon, flin)
    name: str = ""

    @property
    def cells(self) -> int:
        """p-cells (mi+1)(nj+1): the unit of the Mcell-iter/s metric."""
        return (self.mi + 1) * (self.nj + 1)


def add_body(case: Case, shape: int, prm=None, flags: int = 0, t_value: float = 0.0) -> Case:
    """Adds an immersed body's penalty sources (ixb_body_sources, the masks of
    definir_cuerpo, source/mod_front_inmersa.f90:54-179) to case.sources;
    existing sources are kept, so bodies accumulate."""
    mi, nj = case.mi, case.nj
    sh = {0: (mi, nj + 1), 1: (mi + 1, nj), 2: (mi + 1, nj + 1)}
    arrs = {}
    for var in (0, 1, 2):
        if var in case.sources:
            f, l = case.sources[var]
            arrs[var] = (np.array(f, dtype=np.float64, order="F"), np.array(l, dtype=np.float64, order="F"))
        else:
            arrs[var] = (np.zeros(sh[var], order="F"), np.zeros(sh[var], order="F"))
    from ._ffi import check, dptr, lib  # the masks come from the library's ixb_body_sources
    p = None if prm is None else np.ascontiguousarray(prm, dtype=np.float64)
    xp = np.ascontiguousarray(case.xp, dtype=np.float64)
    yp = np.ascontiguousarray(case.yp, dtype=np.float64)
    check(lib.ixb_body_sources(mi, nj, dptr(xp), dptr(yp), shape, None if p is None else dptr(p), flags,
                               float(t_value), dptr(arrs[0][0]), dptr(arrs[0][1]), dptr(arrs[1][0]),
                               dptr(arrs[1][1]), dptr(arrs[2][0]), dptr(arrs[2][1])), "ixb_body_sources")
    for var in (0, 1, 2):
        f, l = arrs[var]
        if var in case.sources or np.any(l != 0.0) or np.any(f != 0.0):
            case.sources[var] = (f, l)
    return case


def shapes(mi: int, nj: int) -> dict:
    return {"u": (mi, nj + 1), "v": (mi + 1, nj), "p": (mi + 1, nj + 1), "T": (mi + 1, nj + 1),
            "u_ant": (mi, nj + 1), "v_ant": (mi + 1, nj), "T_ant": (mi + 1, nj + 1)}


def zero_state(mi: int, nj: int, T0: float = 0.0) -> dict:
    st = {k: np.zeros(s, order="F") for k, s in shapes(mi, nj).items()}
    st["T"][:] = T0
    st["T_ant"][:] = T0
    return st


def default_params(**kw) -> dict:
    p = dict(gamma_momen=0.0, gamma_energ=0.0, Ri=0.0, Riy=0.0, dt=1e30, rel_vel=0.7, rel_pres=0.3,
             rel_ener=0.9, conv_u=1e30, conv_p=1e30, conv_t=1e30, conv_resi=0.0, conv_paso=0.0, p_update=0.6,
             iter_ecuaci_max=0, iter_simple_max=0, solver=0)
    p.update(kw)
    return p


def nondim(adimen: str, Ra: float, Pr: float, Ri_1: float) -> dict:
    """gamma_momen, gamma_energ, Ri, Riy of main.f90:221-244."""
    if adimen == "natural":
        return dict(gamma_momen=math.sqrt(Pr / Ra), gamma_energ=math.sqrt(1.0 / (Pr * Ra)), Ri=0.0, Riy=-1.0)
    if adimen == "mixta":
        return dict(gamma_momen=1.0 / Ra, gamma_energ=1.0 / (Ra * Pr), Ri=0.0, Riy=Ri_1)
    raise ValueError(adimen)


ALL = 1e30  # x1 beyond every node: one segment covers the whole side


def natural_cavity(mi: int = 64, nj: int = 64, Ra: float = 1e4, Pr: float = 0.71, T0: float = 0.5,
                   hot_profile: np.ndarray | None = None, **param_kw) -> Case:
    """Differentially heated square cavity (natural convection): left wall
    T=1, right wall T=0, top and bottom adiabatic, no-slip everywhere,
    zero initial u/v/p and uniform T0."""
    xu, yv, xp, yp = staggered_mesh(mi, nj, "unif", "unif")
    prm = default_params(**nondim("natural", Ra, Pr, 0.0))
    prm.update(param_kw)
    z = [(ALL, BC_DIRI, 0.0)]
    bc = {
        0: bc_table((xu, yp), {0: z, 1: z, 2: z, 3: z}),
        1: bc_table((xp, yv), {0: z, 1: z, 2: z, 3: z}),
        2: bc_table((xp, yp), {0: [(ALL, BC_DIRI, 1.0)], 1: [(ALL, BC_NEUM, 0.0)], 2: [(ALL, BC_DIRI, 0.0)],
                               3: [(ALL, BC_NEUM, 0.0)]}),
    }
    return Case(mi, nj, xu, yv, xp, yp, prm, bc, zero_state(mi, nj, T0), name=f"natural_cavity_{mi}x{nj}_Ra{Ra:g}")


def lid_driven_mixed(mi: int = 701, nj: int = 301, Re: float = 100.0, Ri: float = 1.0, Pr: float = 0.71,
                     beta: float = 1.2, **param_kw) -> Case:
    """Heated lid-driven cavity (mixed convection) on a tanh-clustered mesh:
    lid u=1 on side d, no-slip elsewhere; T=1 on the bottom (side b), T=0
    on the lid (side d), adiabatic side walls.  In 'mixta' mode the reference
    applies buoyancy -Ri*T in +y (Riy = Ri, main.f90:241), so the heated
    wall is the bottom one for a stably stratified cavity."""
    xu, yv, xp, yp = staggered_mesh(mi, nj, "tanh", "tanh", xparam=beta, yparam=beta)
    prm = default_params(**nondim("mixta", Re, Pr, Ri))
    prm.update(param_kw)
    z = [(ALL, BC_DIRI, 0.0)]
    bc = {
        0: bc_table((xu, yp), {0: z, 1: z, 2: z, 3: [(ALL, BC_DIRI, 1.0)]}),
        1: bc_table((xp, yv), {0: z, 1: z, 2: z, 3: z}),
        2: bc_table((xp, yp), {0: [(ALL, BC_NEUM, 0.0)], 1: [(ALL, BC_DIRI, 1.0)], 2: [(ALL, BC_NEUM, 0.0)],
                               3: [(ALL, BC_DIRI, 0.0)]}),
    }
    return Case(mi, nj, xu, yv, xp, yp, prm, bc, zero_state(mi, nj, 0.0), name=f"lid_driven_mixed_{mi}x{nj}_Re{Re:g}")


def lid_driven_forced(mi: int = 256, nj: int = 256, Re: float = 100.0, Pr: float = 0.71, T0: float = 0.5,
                      **param_kw) -> Case:
    """Lid-driven forced convection ('mixta' with Ri = 0, so Ri = Riy = 0 and
    the flow does not depend on T) on a uniform mesh: lid u = 1 on side d,
    no-slip elsewhere; T = 1 on side a (the hot wall; per-line values by
    ixb_set_bc_values), T = 0 on side c, sides b and d adiabatic; zero flow
    and uniform T0 to start."""
    xu, yv, xp, yp = staggered_mesh(mi, nj, "unif", "unif")
    prm = default_params(**nondim("mixta", Re, Pr, 0.0))
    prm.update(param_kw)
    z = [(ALL, BC_DIRI, 0.0)]
    bc = {
        0: bc_table((xu, yp), {0: z, 1: z, 2: z, 3: [(ALL, BC_DIRI, 1.0)]}),
        1: bc_table((xp, yv), {0: z, 1: z, 2: z, 3: z}),
        2: bc_table((xp, yp), {0: [(ALL, BC_DIRI, 1.0)], 1: [(ALL, BC_NEUM, 0.0)], 2: [(ALL, BC_DIRI, 0.0)],
                               3: [(ALL, BC_NEUM, 0.0)]}),
    }
    return Case(mi, nj, xu, yv, xp, yp, prm, bc, zero_state(mi, nj, T0), name=f"lid_driven_forced_{mi}x{nj}_Re{Re:g}")
