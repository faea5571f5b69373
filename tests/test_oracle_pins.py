"""Pins of the CPU oracle against the reference's own known answers.

- test/Doisneau/{MK,IG,AG}: the fields the reference's binary wrote after 5000 iterations of
  its crossing-jets validation cases (tests/golden/crossing_jets_*.npz, made by
  tests/golden/make_golden.py). The reference's gate is L2(rho) <= 1e-4; the oracle is held
  to 1e-12.
- test/Doisneau/IG-chimera: the overlapping-grid variant (two blocks joined by chimera faces,
  102), its density after 5000 iterations (tests/golden/chimera_IG.npz); same gates.
- test/unit/test_muscl_bounds.f90 B1-B5: the bounds of the limited slopes.
- test/unit/test_empty_dt.f90 E1-E7: the steps of empty cells that the coupler's imports fill
  (bound_empty_dt), through a whole step (compute_dt gives the starting steps the unit test sets).
- test/unit/test_radiation.f90 R1-R3: the radiative energy of a cell's source against its closed form.
- test/unit/test_near_empty_cap.f90: the dispersion cap of near-empty IG and AG cells in cons_2_prim.
- test/verification/common.py: every drag and Nusselt correlation against the reference's own Python
  restatement of them (tests/golden/correlations.npz), to 1e-13.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from ice_b200 import abi, configs
from ice_b200.solver import Solver

GOLDEN = Path(__file__).resolve().parent / "golden"
ZERO_AT_NEG = ["vanleer", "mc", "superbee", "koren", "umist", "osher", "sweby", "minmod"]
ALL_LIM = ZERO_AT_NEG + ["vanalbada", "ospre"]


def res_reference_cases():
    """The four crossing-jets cases with the reference's default res-threshold (1e-10), each with the
    first non-zero density residual its binary stored (tests/golden/restart_counters.npz)."""
    g = np.load(GOLDEN / "restart_counters.npz")
    cases = [(lambda cl=cl: configs.crossing_jets(cl, steps=5000), float(g[f"{cl}_ICE_RES_REFERENCE"]))
             for cl in ("MK", "IG", "AG")]
    chim = dict(np.load(GOLDEN / "chimera_IG.npz"))
    cases.append((lambda: configs.doisneau_chimera(chim), float(g["IG_chimera_ICE_RES_REFERENCE"])))
    return cases


def check_res_reference(lib):
    """The unit of res-threshold (Mod_Explicit.f90:222-223), the density residual norm of the first
    step (Mod_Diagnostic.f90:22-83), against the value the reference's binary stored with its
    solutions (ICE_RES_REFERENCE), to 1e-12 relative: the MK case to the last bit, the others to the
    contraction of the reference binary's arithmetic (1.6e-13)."""
    for make, want in res_reference_cases():
        case = make()
        case.numerics.res_threshold = 1e-10
        s = Solver(case, lib)
        assert s.step(1).status == 0
        got = np.zeros(1)
        assert lib.get_res_reference(s.ctx, abi.ptr(got)) == abi.OK
        assert abs(got[0] / want - 1.0) <= 1e-12, (got[0], want)


def test_res_reference_matches_reference_output(orc):
    check_res_reference(orc)


@pytest.mark.slow
def test_chimera_matches_reference_output(orc):
    g = dict(np.load(GOLDEN / "chimera_IG.npz"))
    case = configs.doisneau_chimera(g)
    # every chimera row of the reference's table carries its donors, with weights summing to 1 per layer
    assert len(case.chimera) == int(np.sum(g["bc"][:, 5] == 102)) > 0
    for l1, l2 in case.chimera.values():
        for layer in (l1, l2):
            assert abs(sum(w for *_, w in layer) - 1.0) < 1e-6
    s = Solver(case, orc)
    out = s.step(5000)
    assert out.status == 0 and out.iter == 5000
    for b in range(2):
        p = s.download(b, 0)[2, 2:-2, 2:-2, 0]       # (j, i)
        l2 = math.sqrt(float(np.mean((p - g[f"rho{b + 1}"]) ** 2)))
        assert l2 <= 1e-4                            # the reference's own gate
        assert l2 <= 1e-12, (b, l2)


@pytest.mark.slow
@pytest.mark.parametrize("closure", ["MK", "IG", "AG"])
def test_crossing_jets_matches_reference_output(orc, closure):
    g = np.load(GOLDEN / f"crossing_jets_{closure}.npz")
    case = configs.crossing_jets(closure)
    # the case built here is the reference's: same records, codes and inlet angles
    bc = np.array([(b, i, j, k, f, c, (pay[2] if c == 402 else 0.0)) for (b, i, j, k, f, c, pay) in case.bc_rows])
    assert np.array_equal(bc[:, :6], g["bc"][:, :6])
    assert np.allclose(bc[:, 6], g["bc"][:, 6], rtol=0, atol=0)
    s = Solver(case, orc)
    out = s.step(5000)
    assert out.status == 0 and out.iter == 5000
    p = s.download(0, 0)[2, 2:-2, 2:-2]          # (j, i, v)
    ref = g["field"]                                 # (v, j, i)
    l2 = math.sqrt(float(np.mean((p[..., 0] - ref[0]) ** 2)))
    assert l2 <= 1e-4                                # the reference's own gate
    assert l2 <= 1e-12
    # every field on the occupied cells, relative to the largest value of its group (the velocity
    # components together, the covariance components together)
    occupied = ref[0] > 1e-6
    nc = ref.shape[0]
    groups = [[0], [1, 2, 3]] + ([[4, 5, 6, 7, 8, 9]] if nc == 12 else []) + [[v] for v in range(4 if nc < 12 else 10, nc)]
    for grp in groups:
        scale = max(float(np.abs(ref[grp][:, occupied]).max()), 1e-300)
        for v in grp:
            err = float(np.abs(p[..., v] - ref[v])[occupied].max()) / scale
            assert err <= 1e-9, (closure, v, err)


def _mk_state(q):
    return np.array([1.0, q, 0.0, 0.0, 300.0, 1e8])


def _faces(orc, lim, q, L, beta=1.0):
    pl = np.zeros(12); pr = np.zeros(12)
    st = [_mk_state(x) for x in q]
    args = [abi.ptr(a) for a in st]
    rc = orc.reconstruct(abi.CLOSURE["MK"], abi.LIMITER[lim], *args,
                         0.5 * (L[0] + L[1]), 0.5 * (L[1] + L[2]), 0.5 * (L[2] + L[3]), 0.5 * L[1], 0.5 * L[2],
                         abi.ptr(pl), abi.ptr(pr), beta)
    assert rc == 0
    return pl[1], pr[1]


def _between(v, a, b):
    tol = 8 * np.spacing(max(abs(a), abs(b), np.finfo(float).tiny))
    return min(a, b) - tol <= v <= max(a, b) + tol


@pytest.mark.parametrize("lim", ALL_LIM)
def test_muscl_bounds_B1(orc, lim):
    ul, ur = _faces(orc, lim, [1.0, 0.01, 0.0, 0.0], [1.25, 1.25, 1.0, 1.0])
    assert _between(ul, 0.01, 0.0) and _between(ur, 0.01, 0.0)


@pytest.mark.parametrize("lim", ALL_LIM)
def test_muscl_bounds_B2_random_lines(orc, lim):
    rng = np.random.default_rng(20261110)
    bad_face = bad_slope = 0
    for n in range(2000):
        r = rng.random(10); sg = rng.random(5)
        L = 10.0 ** (2.0 * r[:5]); q = 10.0 ** (6.0 * r[5:] - 3.0)
        monotone = lim not in ZERO_AT_NEG or n % 2 == 1
        if monotone:
            q = np.sort(q)
        else:
            q = np.where(sg > 0.5, -q, q)
        ul, ur = _faces(orc, lim, q[:4], L[:4])
        vl, vr = _faces(orc, lim, q[1:], L[1:])
        if not (_between(ul, q[1], q[2]) and _between(ur, q[1], q[2]) and _between(vl, q[2], q[3]) and _between(vr, q[2], q[3])):
            bad_face += 1
        jump = max(abs(q[2] - q[1]), abs(q[3] - q[2]), np.finfo(float).tiny)
        if abs((vl - q[2]) - (q[2] - ur)) > max(1e-12 * jump, 4 * np.spacing(abs(q[2]))):
            bad_slope += 1
    assert bad_face == 0 and bad_slope == 0


@pytest.mark.parametrize("lim", ALL_LIM)
def test_muscl_bounds_B3_equal_cells_bit_for_bit(orc, lim):
    rng = np.random.default_rng(7)
    big = np.finfo(float).max
    L = abi.LIMITER[lim]
    for _ in range(500):
        q = 2.0 * rng.random(4) - 1.0
        h = 0.01 + rng.random()
        ul, ur = _faces(orc, lim, q, [h, h, h, h])
        s0 = (q[1] - q[0]) / (0.5 * (h + h)); s1 = (q[2] - q[1]) / (0.5 * (h + h)); s2 = (q[3] - q[2]) / (0.5 * (h + h))
        el = q[1] + (orc.limiter(L, s1, s0, big, big) * 1.0) * (0.5 * h)
        er = q[2] - (orc.limiter(L, s2, s1, big, big) * 1.0) * (0.5 * h)
        assert ul == el and ur == er


@pytest.mark.parametrize("lim", ALL_LIM)
def test_muscl_bounds_B4_linear_data_exact(orc, lim):
    rng = np.random.default_rng(11)
    for _ in range(300):
        L = 10.0 ** (2.0 * rng.random(4)); a = 2.0 * rng.random() - 1.0
        x = np.zeros(4)
        x[0] = 0.5 * L[0]
        for m in range(1, 4):
            x[m] = x[m - 1] + 0.5 * (L[m - 1] + L[m])
        xf = x[1] + 0.5 * L[1]
        ul, ur = _faces(orc, lim, a * x, L)
        assert abs(ul - a * xf) <= 1e-12 * abs(a) * x[3] and abs(ur - a * xf) <= 1e-12 * abs(a) * x[3]


@pytest.mark.parametrize("lim", ALL_LIM)
def test_muscl_bounds_B5_injection_side(orc, lim):
    # dll = 0: the left face of the cell sits on its value (an injected ghost)
    pl = np.zeros(12); pr = np.zeros(12)
    st = [_mk_state(x) for x in (0.3, 0.7, 0.2, 0.9)]
    rc = orc.reconstruct(abi.CLOSURE["MK"], abi.LIMITER[lim], *[abi.ptr(a) for a in st],
                         1.0, 1.0, 1.0, 0.0, 0.5, abi.ptr(pl), abi.ptr(pr), 1.0)
    assert rc == 0 and np.isfinite(pl[1]) and np.isfinite(pr[1])
    assert pl[1] == 0.7 or _between(pl[1], 0.7, 0.2)


def test_riemann_1d_runs_and_conserves_mass(orc):
    case = configs.riemann_1d(n=200, steps=50)
    s = Solver(case, orc)
    m0 = float(case.state[0][0][2, 2, 2:-2, 0].sum())
    out = s.step(50)
    assert out.status == 0
    p = s.download(0, 0)[2, 2, 2:-2]
    assert np.isfinite(p).all()
    # the waves have not reached the transmissive ends, where the two streams keep entering:
    # the mass gained per unit section is (rho_L u_L + rho_R |u_R|) t = 1.5 t
    dx = 1.0 / 200
    gained = (float(p[:, 0].sum()) - m0) * dx
    assert abs(gained - 1.5 * out.time) <= 1e-10 * 1.5 * out.time


def _empty_tube_step(orc, n_occupied, source_cell=None, time_accurate=False, narrow_last=False):
    """One step of the unit test's 4-cell tube; returns the step's output and each cell's step."""
    case = configs.empty_tube(n_occupied, time_accurate, narrow_last)
    s = Solver(case, orc)
    if source_cell is not None:
        imp = np.zeros((1, 1, 4, 6))
        imp[0, 0, source_cell - 1] = [2e2, 2e2 * 800.0, 0.0, 0.0, 0.0, 0.0]   # births at 800 m/s
        assert orc.set_imports(s.ctx, 1, 1, abi.ptr(imp)) == 0
    out = s.step(1)
    dt = np.zeros(4)
    orc.download_aux(s.ctx, 1, 1, abi.ptr(dt), None, None)
    return out, dt


def test_empty_dt_unit_cases(orc):
    cfl, dx, dtmax = 0.4, 1e-3, 1e-4
    occ, src = cfl * dx / 100.0, cfl * dx / 800.0
    near = lambda a, b: bool(np.all(np.abs(np.asarray(a) - b) <= 4 * np.finfo(float).eps * abs(b)))
    # E1: no source; the steps compute_dt gives: cfl dx/|u| occupied, the dt-max ceiling empty
    _, dt0 = _empty_tube_step(orc, 2)
    assert near(dt0[:2], occ) and np.all(dt0[2:] == dtmax)
    # E2/E3: imports at 800 m/s into empty cell 3: occupied cells keep their steps, empty ones cfl dx/800
    _, dt = _empty_tube_step(orc, 2, source_cell=3)
    assert np.array_equal(dt[:2], dt0[:2]) and near(dt[2:], src)
    # E4: no occupied cell: every cell at the source's step
    _, dt = _empty_tube_step(orc, 0, source_cell=3)
    assert near(dt, src)
    # E5: a source in occupied cell 1 only: the empty cells at the occupied cells' step
    _, dt = _empty_tube_step(orc, 2, source_cell=1)
    assert np.array_equal(dt[:2], dt0[:2]) and near(dt[2:], occ)
    # E6: the same, empty cell 4 ten times narrower: it steps at its own width at the occupied speed.
    # The unit test sets that cell's metric to 10/dx exactly; here it comes from the nodes 3.0 and
    # 3.1 mm, whose difference is 1e-4 only to a few ulp, so the bound is 64 ulp there
    _, dt = _empty_tube_step(orc, 2, source_cell=1, narrow_last=True)
    assert np.array_equal(dt[:2], dt0[:2]) and near(dt[2:3], occ)
    assert abs(dt[3] - occ / 10.0) <= 64 * np.finfo(float).eps * occ / 10.0
    # E7: time-accurate, imports into empty cell 3, no occupied cell: the global step at the source's
    out, _ = _empty_tube_step(orc, 0, source_cell=3, time_accurate=True)
    assert near([out.dtglobal], src)


def test_imports_are_checked(orc):
    case = configs.empty_tube(2)
    s = Solver(case, orc)
    imp = np.zeros((1, 1, 4, 6))
    assert orc.set_imports(s.ctx, 2, 1, abi.ptr(imp)) == abi.EINVAL
    imp[0, 0, 1, 0] = np.nan
    assert orc.set_imports(s.ctx, 1, 1, abi.ptr(imp)) == abi.EINVAL


def _family(closure, **kw):
    from ice_b200.case import Family
    return Family(closure, **kw).to_c()


def test_radiation_unit_cases(orc):
    """R1-R3: MK drops of 30 um at rest at 2400 K in a gas at rest at 600 K, no drag, no heat, no
    evaporation: the energy slot is eps sigma pi d^2 n (Tg^4 - Tp^4) to 1e-14 at emissivity 0.8, and 0
    at emissivity 0 with every other slot unchanged (R4 needs an emissivity table, which this path
    does not support)."""
    import ctypes as C
    sigma, d, rho_p, tp, tg = 5.670374419e-8, 30e-6, 1.0, 2400.0, 600.0
    rg, gam, kg, mu = 287.05, 1.4, 0.05, 3e-5
    n = rho_p / (2000.0 * math.pi / 6.0 * d ** 3)
    cond = np.array([rho_p, 0.0, 0.0, 0.0, tp, n])
    gas = np.array([101325.0 / (rg * tg), 0.0, 0.0, 0.0, tg])
    out = {}
    for name, em in (("grey", 0.8), ("off", 0.0)):
        fam = _family("MK", rho_al=2000.0, cs_al=1000.0, emiss=em)
        src = np.zeros(6)
        tau = orc.cell_source(abi.CLOSURE["MK"], abi.ptr(cond), abi.ptr(gas), rg, gam, kg, mu, C.byref(fam),
                              abi.DRAG["NoDrag"], abi.HEAT["NoHeat"], 0, abi.ptr(src))
        out[name] = (src, tau)
    q = 0.8 * sigma * math.pi * d * d * n * (tg ** 4 - tp ** 4)
    assert abs(out["grey"][0][4] - q) <= 1e-14 * abs(q)                          # R1
    s8, t8 = out["grey"]
    s0, t0 = out["off"]
    assert s0[4] == 0.0 and np.array_equal(s0[:4], s8[:4]) and s0[5] == s8[5] and t0 == t8    # R2, R3


def test_near_empty_cap_unit_cases(orc):
    import ctypes as C
    cl, t0, eps = 1250.0, 300.0, float(np.float32(1e-25))
    rho_empty, theta_cap = 1e-6, 1.0

    def conv(closure, p):
        fam = _family(closure, rho_al=2950.0, cs_al=cl)
        p = np.array(p, dtype=np.float64)
        c = np.zeros_like(p)
        orc.prim2cons(abi.CLOSURE[closure], abi.ptr(p), abi.ptr(c), C.byref(fam))
        return c

    def back(closure, c):
        fam = _family(closure, rho_al=2950.0, cs_al=cl)
        c = np.array(c, dtype=np.float64)
        q = np.zeros_like(c)
        orc.cons2prim(abi.CLOSURE[closure], abi.ptr(c), abi.ptr(q), C.byref(fam))
        return q

    same_t = lambda t, ref: abs(t - ref) <= 8 * np.spacing(ref)
    # IG (a): 1e-7 kg/m3 at P/rho = 10: P = rho theta_cap exactly, T that of the conservative variables
    rho = 1e-7
    c = conv("IG", [rho, 1.0, 0.5, 0.0, 10 * rho, t0, 1e3])
    q = back("IG", c)
    assert q[4] == q[0] * theta_cap
    assert same_t(q[5], (c[5] - 0.5 * c[4]) / (cl * c[0] + eps)) and same_t(q[5], t0)
    assert q[0] == rho and q[1] == c[1] / (c[0] + eps)
    # (a') at rho_empty itself: capped; (b) 1e-5 (above rho_empty): untouched; below the cap: untouched
    q = back("IG", conv("IG", [rho_empty, 1.0, 0.5, 0.0, 10 * rho_empty, t0, 1e3]))
    assert q[4] == q[0] * theta_cap
    q = back("IG", conv("IG", [1e-5, 1.0, 0.5, 0.0, 1e-4, t0, 1e3]))
    assert abs(q[4] - 1e-4) <= 1e-12 * 1e-4
    q = back("IG", conv("IG", [rho, 1.0, 0.5, 0.0, 0.5 * rho, t0, 1e3]))
    assert abs(q[4] - 0.5 * rho) <= 1e-12 * 0.5 * rho
    # AG (c): 1e-7 kg/m3, trace 30 rho: every component times 3 rho theta_cap / tr = 0.1
    tens = rho * np.array([10.0, 2.0, 1.0, 12.0, 3.0, 8.0])
    c = conv("AG", [rho, 1.0, 0.5, 0.25, *tens, t0, 1e3])
    q = back("AG", c)
    assert np.all(np.abs(q[4:10] - 0.1 * tens) <= 1e-12 * np.abs(tens))
    assert abs(q[4] + q[7] + q[9] - 3 * rho * theta_cap) <= 1e-12 * rho
    assert same_t(q[10], (c[10] - 0.5 * (c[4] + c[7] + c[9])) / (cl * c[0] + eps)) and same_t(q[10], t0)
    p5 = 1e-5 * np.array([10.0, 2.0, 1.0, 12.0, 3.0, 8.0])
    q = back("AG", conv("AG", [1e-5, 1.0, 0.5, 0.25, *p5, t0, 1e3]))
    assert np.all(np.abs(q[4:10] - p5) <= 1e-12 * 1e-4)
    # (d) a NaN second moment stays NaN (the cap is a test, which a NaN fails)
    c = conv("IG", [rho, 1.0, 0.5, 0.0, 10 * rho, t0, 1e3]); c[4] = np.nan
    assert np.isnan(back("IG", c)[4])
    c = conv("AG", [rho, 1.0, 0.5, 0.25, *tens, t0, 1e3]); c[4] = np.nan
    assert np.isnan(back("AG", c)[4])
    # (e) a negative density: the floor overwrites every primitive, all finite
    c = conv("AG", [1e-7, 1.0, 0.5, 0.25, *tens, t0, 1e3]); c[0] = -1e-10
    q = back("AG", c)
    assert np.all(np.isfinite(q)) and np.all(q[4:10] >= 0.0) and q[5] == 0.0 and q[0] > 0.0


def test_correlations_match_reference_restatement(orc):
    g = np.load(GOLDEN / "correlations.npz")
    Re, Ma, Tr, Pr, G = g["Re"], g["Ma"], g["Tr"], g["Pr"], float(g["G"])
    for key in g.files:
        if key.startswith("cd_"):
            sel = abi.DRAG[key[3:]]
            got = np.array([[[orc.drag(r, m, G, t, sel) for t in Tr] for m in Ma] for r in Re])
        elif key.startswith("nu_"):
            sel = abi.HEAT[key[3:]]
            got = np.array([[[orc.heat(r, p, m, sel) for m in Ma] for p in Pr] for r in Re])
        else:
            continue
        ref = g[key]
        assert np.all(np.abs(got - ref) <= 1e-13 * np.abs(ref)), key
