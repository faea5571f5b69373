"""The driver stand-in's set-up: a multi-block mesh with its metrics, the boundary
table, the frozen gas and the initial state, in the layouts the ABI takes.

In ICE this is the work of the Fortran driver before the solve stage
(Wrap_Setup.f90:9-121): read_ic, setup_metrics, Setup_BC + Pair_Connections,
setup_gas, setup_cond. The metric restatement follows
src/lib/numerics/space/Mod_Metrics.f90 (extrapolate_nodes 461-498, normal_signs
503-546, compute_metrics 549-680, compute_metric_tensor 693-779); pairing is the
library's own ice_gpu_pair_connections.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi

GUIDE = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]])

MESH_FIT = 1e-2     # node planes match a turn or a translation to this fraction of a block's thickness
MESH_ANGLE = 1e-6   # a node this close to the x axis, relative to the farthest, has no azimuth
MIRROR = (200, 300, 301)


class SetupError(ValueError):
    """A case the reference's set-up stops on."""


def _thickness(nodes, d):
    """The largest move of a node from node plane 0 to plane 1 of direction d (1 = j, 2 = k), over the three
    coordinates (Mod_Metrics.f90:286-303)."""
    a, b = (nodes[:, 0], nodes[:, 1]) if d == 1 else (nodes[:, :, 0], nodes[:, :, 1])
    return float(np.abs(b - a).max())


def _plane_fit(nodes, d, delthe):
    """How far the node planes 0 and 1 of direction d lie from the mirror planes they should be, over the
    thickness of the block: planes normal to y (d = 1) or z (d = 2), or, on a wedge of angle delthe, the
    planes through the x axis at -/+ delthe/2 (Mod_Metrics.f90:312-355)."""
    thick = _thickness(nodes, d)
    off = 0.0
    for s in (0, 1):
        if d == 1:
            pl = nodes[:, s, :, 1]
            off = max(off, float(np.abs(pl - pl[0, 0]).max()))
        elif delthe == 0.0:
            pl = nodes[:, :, s, 2]
            off = max(off, float(np.abs(pl - pl[0, 0]).max()))
        else:
            ang = (s - 0.5) * delthe
            pl = nodes[:, :, s]
            off = max(off, float(np.abs(pl[..., 2] * np.cos(ang) - pl[..., 1] * np.sin(ang)).max()))
    return off / thick if thick > 0.0 else np.inf


# --------------------------------------------------------------------- metrics
def _cross(u, v):
    return np.stack([u[..., 1] * v[..., 2] - u[..., 2] * v[..., 1],
                     u[..., 2] * v[..., 0] - u[..., 0] * v[..., 2],
                     u[..., 0] * v[..., 1] - u[..., 1] * v[..., 0]], axis=-1)


class Geometry:
    """Metrics of one block from its nodes.

    nodes: (ni+1, nj+1, nk+1, 3) node coordinates (index order i, j, k).
    Output arrays are in the ABI's Fortran layouts, i fastest.
    """

    def __init__(self, nodes: np.ndarray):
        ni, nj, nk = (s - 1 for s in nodes.shape[:3])
        self.dims = (ni, nj, nk)
        X = np.zeros((ni + 3, nj + 3, nk + 3, 3))          # node(-1:ni+1, ...) at [i+1]
        X[1:ni + 2, 1:nj + 2, 1:nk + 2] = nodes
        # extrapolate_nodes (plane meshes): N(-1) = 2 N(0) - N(1)
        X[0, 1:nj + 2, 1:nk + 2] = 2.0 * X[1, 1:nj + 2, 1:nk + 2] - X[2, 1:nj + 2, 1:nk + 2]
        X[ni + 2, 1:nj + 2, 1:nk + 2] = 2.0 * X[ni + 1, 1:nj + 2, 1:nk + 2] - X[ni, 1:nj + 2, 1:nk + 2]
        X[:, 0, 1:nk + 2] = 2.0 * X[:, 1, 1:nk + 2] - X[:, 2, 1:nk + 2]
        X[:, nj + 2, 1:nk + 2] = 2.0 * X[:, nj + 1, 1:nk + 2] - X[:, nj, 1:nk + 2]
        X[:, :, 0] = 2.0 * X[:, :, 1] - X[:, :, 2]
        X[:, :, nk + 2] = 2.0 * X[:, :, nk + 1] - X[:, :, nk]
        self._X = X

        def nd(i, j, k):  # node(i,j,k) with i in -1..ni+1 (scalar or slice-offset arrays)
            return X[i + 1, j + 1, k + 1]

        # normal_signs from the first cell
        def sgn_dir(d1, d2, c1, c2):
            d3 = _cross(d1, d2)
            return 1.0 if np.dot(c1 - c2, d3) >= 0 else -1.0
        n = lambda i, j, k: nd(i, j, k)
        si = sgn_dir(n(1, 1, 1) - n(1, 0, 0), n(1, 0, 1) - n(1, 1, 0),
                     0.25 * (n(1, 1, 1) + n(1, 0, 1) + n(1, 0, 0) + n(1, 1, 0)),
                     0.25 * (n(0, 1, 1) + n(0, 0, 1) + n(0, 0, 0) + n(0, 1, 0)))
        sj = sgn_dir(n(0, 1, 1) - n(1, 1, 0), n(1, 1, 1) - n(0, 1, 0),
                     0.25 * (n(1, 1, 1) + n(0, 1, 1) + n(0, 1, 0) + n(1, 1, 0)),
                     0.25 * (n(1, 0, 1) + n(0, 0, 1) + n(0, 0, 0) + n(1, 0, 0)))
        sk = sgn_dir(n(0, 1, 1) - n(1, 0, 1), n(0, 0, 1) - n(1, 1, 1),
                     0.25 * (n(1, 1, 1) + n(0, 1, 1) + n(0, 0, 1) + n(1, 0, 1)),
                     0.25 * (n(1, 1, 0) + n(0, 1, 0) + n(0, 0, 0) + n(1, 0, 0)))

        def sl(lo, hi):
            return slice(lo + 1, hi + 2)

        def faces(d1, d2, s):
            d3 = _cross(d1, d2) * 0.5
            A = np.sqrt(d3[..., 0] * d3[..., 0] + d3[..., 1] * d3[..., 1] + d3[..., 2] * d3[..., 2])
            with np.errstate(invalid="ignore", divide="ignore"):
                N = np.where(A[..., None] == 0.0, 0.0, d3 / A[..., None] * s)
            return np.concatenate([N, A[..., None]], axis=-1)

        # i faces: i = 0..ni, j = 1..nj, k = 1..nk  (arrays indexed [i, j, k])
        I0, I1 = sl(0, ni), sl(-1, ni - 1)
        J0, J1 = sl(1, nj), sl(0, nj - 1)
        K0, K1 = sl(1, nk), sl(0, nk - 1)
        f1 = faces(X[I0, J0, K0] - X[I0, J1, K1], X[I0, J1, K0] - X[I0, J0, K1], si)
        # j faces: i = 1..ni, j = 0..nj, k = 1..nk
        I0, I1 = sl(1, ni), sl(0, ni - 1)
        J0 = sl(0, nj)
        f2 = faces(X[I1, J0, K0] - X[I0, J0, K1], X[I0, J0, K0] - X[I1, J0, K1], sj)
        # k faces: i = 1..ni, j = 1..nj, k = 0..nk
        J0, J1 = sl(1, nj), sl(0, nj - 1)
        K0 = sl(0, nk)
        f3 = faces(X[I1, J0, K0] - X[I0, J1, K0], X[I1, J1, K0] - X[I0, J0, K0], sk)
        self.face = [np.ascontiguousarray(f.transpose(2, 1, 0, 3)) for f in (f1, f2, f3)]

        # volumes (the exact trilinear integral)
        c0 = X[sl(0, ni - 1), sl(0, nj - 1), sl(0, nk - 1)]
        r = [None] * 9
        for a in (0, 1):
            for b in (0, 1):
                for cc in (0, 1):
                    q = 1 + a + 2 * b + 4 * cc
                    r[q] = X[sl(a, ni - 1 + a), sl(b, nj - 1 + b), sl(cc, nk - 1 + cc)] - c0
        ea1 = 0.25 * (r[2] + (r[6] - r[5]) + (r[4] - r[3]) + (r[8] - r[7]))
        ea2 = 0.25 * (r[3] + (r[7] - r[5]) + (r[4] - r[2]) + (r[8] - r[6]))
        ea3 = 0.25 * (r[5] + (r[7] - r[3]) + (r[6] - r[2]) + (r[8] - r[4]))
        dot = lambda u, v: (u * v).sum(-1)
        vol = dot(ea1, _cross(r[7], r[5] - r[3]) + _cross(r[8] - r[2], r[6] - r[4]))
        vol = vol + dot(ea2, _cross(r[6], r[2] - r[5]) + _cross(r[8] - r[3], r[4] - r[7]))
        vol = vol + dot(ea3, _cross(r[4], r[3] - r[2]) + _cross(r[8] - r[5], r[7] - r[6]))
        vol = np.abs(vol / 12.0)
        self.vol = np.ascontiguousarray(vol.transpose(2, 1, 0))

        # metric tensor and mean lengths on 0..n+1
        P = lambda a, b, cc: X[a:a + ni + 2, b:b + nj + 2, cc:cc + nk + 2]   # node(i-1+a, ...) for i=0..ni+1
        # node(i,j,k) at offset (1,1,1) relative to node(i-1,j-1,k-1) at (0,0,0)
        # left to right, as the Fortran sums are written
        A1 = P(1, 1, 1) - P(0, 1, 1) + P(1, 0, 1) - P(0, 0, 1) + P(1, 1, 0) - P(0, 1, 0) + P(1, 0, 0) - P(0, 0, 0)
        A2 = P(1, 1, 1) - P(1, 0, 1) + P(0, 1, 1) - P(0, 0, 1) + P(1, 1, 0) - P(1, 0, 0) + P(0, 1, 0) - P(0, 0, 0)
        A3 = P(1, 1, 1) - P(1, 1, 0) + P(0, 1, 1) - P(0, 1, 0) + P(1, 0, 1) - P(1, 0, 0) + P(0, 0, 1) - P(0, 0, 0)
        A = 0.25 * np.stack([A1, A2, A3], axis=-2)          # A[..., row, col]
        det = (A[..., 0, 0] * A[..., 1, 1] * A[..., 2, 2] - A[..., 0, 0] * A[..., 1, 2] * A[..., 2, 1]
               - A[..., 0, 1] * A[..., 1, 0] * A[..., 2, 2] + A[..., 0, 1] * A[..., 1, 2] * A[..., 2, 0]
               + A[..., 0, 2] * A[..., 1, 0] * A[..., 2, 1] - A[..., 0, 2] * A[..., 1, 1] * A[..., 2, 0])
        cof = np.empty_like(A)
        cof[..., 0, 0] = (A[..., 1, 1] * A[..., 2, 2] - A[..., 1, 2] * A[..., 2, 1])
        cof[..., 0, 1] = -(A[..., 1, 0] * A[..., 2, 2] - A[..., 1, 2] * A[..., 2, 0])
        cof[..., 0, 2] = (A[..., 1, 0] * A[..., 2, 1] - A[..., 1, 1] * A[..., 2, 0])
        cof[..., 1, 0] = -(A[..., 0, 1] * A[..., 2, 2] - A[..., 0, 2] * A[..., 2, 1])
        cof[..., 1, 1] = (A[..., 0, 0] * A[..., 2, 2] - A[..., 0, 2] * A[..., 2, 0])
        cof[..., 1, 2] = -(A[..., 0, 0] * A[..., 2, 1] - A[..., 0, 1] * A[..., 2, 0])
        cof[..., 2, 0] = (A[..., 0, 1] * A[..., 1, 2] - A[..., 0, 2] * A[..., 1, 1])
        cof[..., 2, 1] = -(A[..., 0, 0] * A[..., 1, 2] - A[..., 0, 2] * A[..., 1, 0])
        cof[..., 2, 2] = (A[..., 0, 0] * A[..., 1, 1] - A[..., 0, 1] * A[..., 1, 0])
        with np.errstate(invalid="ignore", divide="ignore"):
            M = np.where((np.abs(det) == 0.0)[..., None, None], np.eye(3), cof / det[..., None, None])
        dl = np.sqrt(A[..., 0] ** 2 + A[..., 1] ** 2 + A[..., 2] ** 2)     # |row h|
        # Fortran c(3,3) is column-major: flat index 3*col + row
        self.M = np.ascontiguousarray(M.transpose(2, 1, 0, 4, 3).reshape(nk + 2, nj + 2, ni + 2, 9))
        self.dl = np.ascontiguousarray(dl.transpose(2, 1, 0, 3))


def box_nodes(ni, nj, nk, lo=(0.0, 0.0, 0.0), size=(1.0, 1.0, 1.0)):
    x = np.linspace(lo[0], lo[0] + size[0], ni + 1)
    y = np.linspace(lo[1], lo[1] + size[1], nj + 1)
    z = np.linspace(lo[2], lo[2] + size[2], nk + 1)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    return np.stack([X, Y, Z], axis=-1)


# ------------------------------------------------------------------ the case
@dataclass
class Family:
    closure: str
    riemann: str = ""                 # '' = the reference's default per closure
    rho_al: float = 2700.0
    cs_al: float = 1598.0
    lv_al: float = 1.08e7
    emiss: float = 0.0
    evap: str = "none"
    intf: str = "VLE"
    Mv: float = 26.98
    cpv: float = 0.0
    Le: float = 1.0
    Yinf: float = 0.0
    Tboil: float = 2792.0
    alphaE: float = 1.0
    frozen: tuple = ()

    @property
    def nc(self):
        return abi.NBASE[abi.CLOSURE[self.closure]]

    def to_c(self) -> abi.Family:
        f = abi.Family()
        f.closure = abi.CLOSURE[self.closure]
        r = self.riemann or ("Saurel" if self.closure == "MK" else "Rusanov")
        f.riemann = abi.RIEMANN[r]
        f.nfrozen = len(self.frozen)
        for q, s in enumerate(self.frozen):
            f.frozen[q] = s
        f.rho_al, f.cs_al, f.lv_al, f.emiss = self.rho_al, self.cs_al, self.lv_al, self.emiss
        f.evap = abi.EVAP[self.evap]
        f.intf = 1 if self.intf == "LK" else 0
        f.liq = 0
        f.boil = 0
        Ru = 8314.46
        ep = [self.Mv, self.lv_al, self.cpv, self.Le, self.Yinf, self.lv_al * self.Mv / Ru, 1.0 / self.Tboil,
              self.alphaE]
        for q, v in enumerate(ep):
            f.ep[q] = v
        return f


@dataclass
class Numerics:
    scheme: str = "RK2"
    time_accurate: bool = True
    cfl: float = 0.5
    dt_max: float = 1e-4
    tau_factor: float = 1.0
    cfl_ramp_iter: int = 0
    limiter: str = "vanleer"          # 'IORD' = first order
    shock_detector: bool = False
    irs: bool = False
    irs_beta: float = 0.5
    coupled: bool = False
    drag: str = "Schiller-Naumann"
    heat: str = "Ranz-Marshall"
    blowing: bool = False
    precision: int = abi.PREC_FP64
    realize: bool = True              # the FP32-flux form's realizability correction of AG states
    itermax: int = 1_000_000_000
    time_threshold: float = 1e30
    res_threshold: float = 0.0
    sol_diter: int = 0                # a solution every sol_diter iterations (0: at the end only)


@dataclass
class Case:
    """Everything the driver hands the solve stage."""
    name: str
    nodes: list                       # per block (ni+1, nj+1, nk+1, 3)
    families: list                    # of Family
    numerics: Numerics
    bc_rows: list                     # one copy of the table: (b,i,j,k,f,code, payload tuple)
    state: list = field(default_factory=list)   # per block, per family: (nk+4,nj+4,ni+4,nc)
    gas: list = field(default_factory=list)     # per block: dict prim5,R,gam,k,mu
    geoms: list = field(default_factory=list)
    rec_int: np.ndarray = None
    rec_real: np.ndarray = None
    # chimera (102) rows of bc_rows: row number -> (donors of ghost layer 1, donors of layer 2), each a
    # list of (b, i, j, k, weight) as the case's boundary file lists them (IO_BC.f90:209-236)
    chimera: dict = field(default_factory=dict)
    chim_n: np.ndarray = None
    chim_donor: np.ndarray = None
    chim_weight: np.ndarray = None
    # per-family copies of the table (ATLAS writes one copy per population, each with its own inlet
    # data; copy c drives family c): None, one copy (it speaks for every family) or one per family.
    # Every copy lists the same rows; only the inlet payloads differ.
    bc_copies: list = None

    @property
    def dims(self):
        return [tuple(s - 1 for s in n.shape[:3]) for n in self.nodes]

    @property
    def ndir(self):
        d = 1
        for (ni, nj, nk) in self.dims:
            if nj > 1:
                d = max(d, 2)
            if nk > 1:
                d = 3
        return d

    def wedge_angle(self) -> float:
        """check_mesh_type (Mod_Metrics.f90:103-176): on a 2-D mesh, the angle of the axisymmetric wedge when in
        every block the k = 1 node plane is the k = 0 plane turned about the x axis by one angle, 0 when it
        is the k = 0 plane translated; misfits are measured against the block's thickness. A block that is
        neither, wedges of different angles, and wedge blocks beside plane ones stop the set-up."""
        if self.ndir != 2:
            return 0.0
        rmax = max(float(np.hypot(n[..., 1], n[..., 2]).max()) for n in self.nodes)
        angles = []
        for b, n in enumerate(self.nodes):
            p0, p1 = n[:, :, 0], n[:, :, 1]
            thick = _thickness(n, 2)
            move = p1 - p0
            fit_move = float(np.abs(move - move[0, 0]).max()) / thick
            r0 = np.hypot(p0[..., 1], p0[..., 2])
            far = r0 > MESH_ANGLE * rmax
            fit_turn, ang = np.inf, 0.0
            if far.any():
                turn = np.arctan2(p1[..., 2], p1[..., 1]) - np.arctan2(p0[..., 2], p0[..., 1])
                ang = float(np.median(turn[far]))
                c, s_ = np.cos(ang), np.sin(ang)
                rot = np.stack([p0[..., 0], c * p0[..., 1] - s_ * p0[..., 2], s_ * p0[..., 1] + c * p0[..., 2]], axis=-1)
                fit_turn = float(np.abs(p1 - rot).max()) / thick
            turned = fit_turn <= MESH_FIT and fit_turn < fit_move and abs(ang) > MESH_ANGLE
            moved = fit_move <= MESH_FIT and not turned
            if not (turned or moved):
                raise SetupError(f"block {b + 1}: its k = 1 node plane is neither the k = 0 plane turned about the x "
                                 f"axis nor translated (the turn fits to {fit_turn:.2e} of its thickness, the "
                                 f"translation to {fit_move:.2e})")
            angles.append(ang if turned else None)
        turned = [a for a in angles if a is not None]
        if not turned:
            return 0.0
        if len(turned) != len(angles):
            raise SetupError(f"{len(turned)} of the {len(angles)} blocks of the 2-D mesh are axisymmetric wedges, "
                             "the others plane")
        if any(abs(a - turned[0]) > MESH_FIT * abs(turned[0]) for a in turned):
            raise SetupError("the blocks of the 2-D mesh are wedges of different angles")
        return turned[0]

    def setup_freeze(self):
        """setup_freeze (Mod_Freeze.f90:30-140): between two faces that mirror the flow one cell apart (the k
        faces of a 2-D mesh, the j and k faces of a 1-D one) the components odd across them have a mode the
        time step does not resolve; they are set to zero here and not integrated (the families' frozen
        slots, which zero their source and residual). w across mirror k faces that are planes normal to z,
        or on an axisymmetric wedge (whose k faces must all be 200); v across mirror j faces normal to y on
        a 1-D mesh; with AG also P13 (w), P12 (v) and P23 (either). Returns the reference's warning, or
        None when nothing is frozen."""
        ndir, delthe = self.ndir, self.wedge_angle()
        nj = nk = nmj = nmk = 0
        other = None
        for (b, i, j, k, f, code, _pay) in self.bc_rows:
            if f in (3, 4):
                nj += 1
                nmj += code in MIRROR
            elif f in (5, 6):
                nk += 1
                nmk += code in MIRROR
                if code != 200 and other is None:
                    other = (b, i, j, f, code)
        freeze_v = freeze_w = False
        if ndir == 2 and delthe != 0.0:
            if other is not None:
                b, i, j, f, code = other
                raise SetupError(f"face {f} of the cell (block i j) {b} {i} {j} carries {code}: the k faces of an "
                                 "axisymmetric wedge must carry 200, the mirror that keeps the flow axisymmetric")
            if max(_plane_fit(n, 2, delthe) for n in self.nodes) > MESH_FIT:
                raise SetupError("the k node planes of the axisymmetric wedge are not the planes at -/+ delthe/2 "
                                 "about z = 0: the wedge must be symmetric about the plane z = 0")
            freeze_w = True
        elif ndir <= 2:
            if nk > 0 and nmk == nk:
                freeze_w = max(_plane_fit(n, 2, 0.0) for n in self.nodes) <= MESH_FIT
            if ndir == 1 and nj > 0 and nmj == nj:
                freeze_v = max(_plane_fit(n, 1, 0.0) for n in self.nodes) <= MESH_FIT
        for p, fam in enumerate(self.families):
            odd = {3: freeze_v, 4: freeze_w}
            if fam.closure == "AG":
                odd.update({6: freeze_v, 7: freeze_w, 9: freeze_v or freeze_w})
            fam.frozen = tuple(sorted(slot for slot, on in odd.items() if on))
            for per_fam in self.state:
                for slot in fam.frozen:
                    per_fam[p][..., slot - 1] = 0.0
        if not (freeze_v or freeze_w):
            return None
        ag = any(f.closure == "AG" for f in self.families)
        if freeze_v and freeze_w:
            what, faces = ("v and w (with AG also P12, P13 and P23)" if ag else "v and w"), "j and k"
        elif freeze_v:
            what, faces = ("v (with AG also P12 and P23)" if ag else "v"), "j"
        else:
            what, faces = ("w (with AG also P13 and P23)" if ag else "w"), "k"
        if ndir == 2 and delthe != 0.0:
            return f"axisymmetric wedge: the swirl {what} set to zero and not integrated"
        return f"{'2-D plane' if ndir == 2 else '1-D'} mesh with mirror {faces} faces: {what} set to zero and not integrated"

    @property
    def ncells(self):
        return int(sum(a * b * c for a, b, c in self.dims))

    def params(self) -> abi.Params:
        nm = self.numerics
        P = abi.Params()
        P.nfam = len(self.families)
        P.ndir = self.ndir
        P.nrk = {"euler": 1, "RK2": 2, "RK3": 3}[nm.scheme]
        P.time_accurate = int(nm.time_accurate)
        P.cfl, P.dt_max, P.tau_factor = nm.cfl, nm.dt_max, nm.tau_factor
        P.cfl_ramp_iter = nm.cfl_ramp_iter
        P.limiter = abi.LIMITER[nm.limiter]
        P.shock_detector = int(nm.shock_detector)
        P.irs, P.irs_beta = int(nm.irs), nm.irs_beta
        P.coupled = int(nm.coupled)
        P.drag, P.heat, P.blow = abi.DRAG[nm.drag], abi.HEAT[nm.heat], int(nm.blowing)
        P.precision = nm.precision
        P.no_realize = 0 if nm.realize else 1
        P.itermax = nm.itermax
        P.sol_diter, P.shell_diter, P.res_diter = nm.sol_diter, 0, 0
        P.time_threshold, P.res_threshold, P.sol_dtime = nm.time_threshold, nm.res_threshold, 1e30
        for p, f in enumerate(self.families):
            P.fam[p] = f.to_c()
        return P

    # ----------------------------------------------------------- set-up work
    def build_geometry(self):
        self.geoms = [Geometry(n) for n in self.nodes]

    def build_records(self, lib: abi.Backend):
        """The records of every family, record n of family p at n * nfam + p: one copy of the table
        speaks for every family, one copy per family (bc_copies) each for its own, any other count stops
        the set-up (IO_BC.f90:290-320); then the connections paired by the library's
        ice_gpu_pair_connections."""
        ng = len(self.families)
        nrow = len(self.bc_rows)
        copies = [self.bc_rows] * ng
        if self.bc_copies is not None:
            if len(self.bc_copies) not in (1, ng):
                raise SetupError(f"{len(self.bc_copies)} copies of the boundary table for {ng} families: one "
                                 "copy speaks for every family, else one copy per family")
            copies = list(self.bc_copies) * (ng if len(self.bc_copies) == 1 else 1)
            for c, rows in enumerate(copies):
                if len(rows) != nrow or any(r[:6] != q[:6] for r, q in zip(rows, self.bc_rows)):
                    raise SetupError(f"copy {c + 1} of the boundary table does not list the rows of the first")
        ri = np.zeros((nrow * ng, abi.REC_INTS), dtype=np.int32)
        rr = np.zeros((nrow * ng, abi.REC_REALS), dtype=np.float64)
        for n in range(nrow):
            for p in range(ng):
                b, i, j, k, f, code, pay = copies[p][n]
                idx = n * ng + p
                ri[idx, :7] = (b, i, j, k, f, code, p + 1)
                if code in (101, 201):
                    ri[idx, 7:12] = pay[:5]
                elif 401 <= code <= 403:
                    rr[idx, :len(pay)] = pay
        if self.chimera:
            cn = np.zeros((nrow * ng, 2), dtype=np.int32)
            don, wts = [], []
            for n in range(nrow):
                l1, l2 = self.chimera.get(n, ((), ()))
                for p in range(ng):
                    cn[n * ng + p] = (len(l1), len(l2))
                    for (b, i, j, k, w) in list(l1) + list(l2):
                        don.append((b, i, j, k)); wts.append(w)
            self.chim_n = cn
            self.chim_donor = np.array(don, dtype=np.int32).reshape(-1, 4)
            self.chim_weight = np.array(wts, dtype=np.float64)
        dims = np.array(self.dims, dtype=np.int32).reshape(-1)
        err = C.create_string_buffer(512)
        rc = lib.pair_connections(len(self.nodes), abi.ptr(dims, C.c_int32), ng, ri.shape[0],
                                  abi.ptr(ri, C.c_int32), err, 512)
        if rc != 0:
            raise ValueError("pairing failed: " + err.value.decode())
        self.rec_int, self.rec_real = ri, rr


def empty_state(dims, nc, fill=np.nan):
    ni, nj, nk = dims
    return np.full((nk + 4, nj + 4, ni + 4, nc), fill)


def interior(a):
    return a[2:-2, 2:-2, 2:-2]


def box_bc(b, dims, codes, payload=None, face_major=False):
    """One block's boundary table. Default: the order of the reference's bench generator
    (test/bench/make_case.py: i faces per (j,k), then j faces, then k faces); face_major: face 1,
    then 2, ... 6, each face's cells with the first index fastest (the ATLAS tables of the
    reference's validation cases). codes: {face: code}; payload(face, i, j, k) -> tuple."""
    ni, nj, nk = dims
    rows = []

    def rec(i, j, k, f):
        code = codes[f]
        pay = payload(f, i, j, k) if (payload and 401 <= code <= 403) else ()
        rows.append((b, i, j, k, f, code, pay))
    if face_major:
        for f in range(1, 7):
            d = (f - 1) // 2
            n = [ni, nj, nk]
            fixed = 1 if f % 2 == 1 else n[d]
            t1, t2 = [a for a in range(3) if a != d]
            for c2 in range(1, n[t2] + 1):
                for c1 in range(1, n[t1] + 1):
                    ijk = [0, 0, 0]
                    ijk[d], ijk[t1], ijk[t2] = fixed, c1, c2
                    rec(ijk[0], ijk[1], ijk[2], f)
        return rows
    for k in range(1, nk + 1):
        for j in range(1, nj + 1):
            rec(1, j, k, 1)
            rec(ni, j, k, 2)
    for k in range(1, nk + 1):
        for i in range(1, ni + 1):
            rec(i, 1, k, 3)
            rec(i, nj, k, 4)
    for j in range(1, nj + 1):
        for i in range(1, ni + 1):
            rec(i, j, 1, 5)
            rec(i, j, nk, 6)
    return rows
