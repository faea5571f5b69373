"""Riemann problems of the anisotropic Gaussian (AG) closure against exact solutions, on the oracle and on
the CUDA path: the reference's Berthon cases (test/Berthon/{SCS,RCS,RCR,SCS-hlle}, checked by its
berthon.py against the tabulated wave patterns of Results/<case>/<case>_exact.tec) and its anisotropic
Sod tube (test/Riemann/AG/verify.py, against the exact gamma = 3 Riemann solution of the 1-D system).
The initial states, thresholds, tolerances and exact profiles are the reference's, in
tests/golden/ag_riemann.npz (made by tests/golden/make_golden.py)."""
import math
from pathlib import Path

import numpy as np
import pytest

from ice_b200 import configs
from ice_b200.solver import Solver

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "ag_riemann.npz")


def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from ice_b200 import abi
    return abi.load_gpu()


def _run(case, lib, t_end, cap=100000):
    """Steps until the time reaches t_end, as the reference's time-threshold stop does."""
    s = Solver(case, lib)
    out = s.step(1)
    while out.time < t_end * (1.0 - 1e-12):
        assert out.iter < cap
        out = s.step(1)
    assert out.status == 0
    return out.time, s.download(0, 0)[2, 2:-2, 2:-2]


def _profile(xy, x):
    """A piecewise-linear profile at x; a repeated abscissa is a jump (berthon.py: sample)."""
    xe, ve = xy
    out = np.empty_like(x)
    for c, xc in enumerate(x):
        if xc <= xe[0]:
            out[c] = ve[0]
            continue
        out[c] = ve[-1]
        for i in range(len(xe) - 1):
            if xe[i] <= xc <= xe[i + 1] and xe[i + 1] > xe[i]:
                out[c] = ve[i] + (ve[i + 1] - ve[i]) * (xc - xe[i]) / (xe[i + 1] - xe[i])
                break
    return out


def _berthon_checks(lib, name):
    """The L1 error of density, u, v, P11, P22 and det P = P11 P22 - P12^2 over the cells, divided by the
    number of cells and the span of the exact profile, within the case's tolerance (berthon.py: verify)."""
    key = name.replace("-", "_")
    ic, x, t_end = GOLD[key + "_ic"], GOLD[key + "_x"], float(GOLD[key + "_t"])
    case = configs.ag_tube(ic, x0=float(x[0]), lx=float(x[-1] - x[0]), t_end=t_end,
                           riemann="HLLE" if bool(GOLD[key + "_hlle"]) else "Rusanov")
    _, p = _run(case, lib, t_end)
    q = p[0]
    nx = q.shape[0]
    xc = x[0] + (np.arange(nx) + 0.5) * (x[-1] - x[0]) / nx
    fields = (q[:, 0], q[:, 1], q[:, 2], q[:, 4], q[:, 7], q[:, 4] * q[:, 7] - q[:, 5] ** 2)
    errors = []
    for z, num in enumerate(fields):
        exact = GOLD[f"{key}_exact{z}"]
        ref = _profile(exact, xc)
        errors.append(float(np.abs(num - ref).sum() / (nx * (exact[1].max() - exact[1].min()))))
    assert max(errors) <= float(GOLD[key + "_tol"]), errors
    return errors


def exact_riemann(left, right, gamma):
    """The exact Riemann solution of the gamma-law Euler equations for W = (rho, u, p), by the method of
    Toro (Riemann Solvers and Numerical Methods for Fluid Dynamics, ch. 4): Newton iteration on the
    pressure function f_L(p) + f_R(p) + u_R - u_L = 0, then the wave pattern sampled along x/t.
    Returns p*, u* and a function of the similarity variable S giving (rho, u, p) arrays."""
    g = gamma

    def side(p, w):
        rho, _, pk = w
        c = math.sqrt(g * pk / rho)
        if p > pk:                                   # shock branch
            a, b = 2.0 / ((g + 1.0) * rho), (g - 1.0) / (g + 1.0) * pk
            root = math.sqrt(a / (p + b))
            return (p - pk) * root, root * (1.0 - 0.5 * (p - pk) / (b + p))
        ratio = p / pk                               # rarefaction branch
        return (2.0 * c / (g - 1.0) * (ratio ** ((g - 1.0) / (2.0 * g)) - 1.0),
                ratio ** (-(g + 1.0) / (2.0 * g)) / (rho * c))

    p = 0.5 * (left[2] + right[2])
    for _ in range(100):
        fl, dl = side(p, left)
        fr, dr = side(p, right)
        step = (fl + fr + right[1] - left[1]) / (dl + dr)
        p_new = max(p - step, 1e-12 * p)
        converged = abs(p_new - p) <= 1e-15 * 0.5 * (p_new + p)
        p = p_new
        if converged:
            break
    u = 0.5 * (left[1] + right[1]) + 0.5 * (side(p, right)[0] - side(p, left)[0])

    def state(s, w, sign):
        """The solution at S on one side of the contact; sign -1 left, +1 right. In the frame mirrored
        for the right side (u -> -u, S -> -S) both sides read as the left one."""
        rho, uk, pk = w[0], sign * -w[1], w[2]
        ss, us = sign * -s, sign * -u
        c = math.sqrt(g * pk / rho)
        if p > pk:
            speed = uk - c * math.sqrt((g + 1.0) / (2.0 * g) * p / pk + (g - 1.0) / (2.0 * g))
            if ss <= speed:
                return rho, w[1], pk
            r = (g - 1.0) / (g + 1.0)
            return rho * (p / pk + r) / (r * p / pk + 1.0), u, p
        head, tail = uk - c, us - c * (p / pk) ** ((g - 1.0) / (2.0 * g))
        if ss <= head:
            return rho, w[1], pk
        if ss > tail:
            return rho * (p / pk) ** (1.0 / g), u, p
        base = 2.0 / (g + 1.0) + (g - 1.0) / ((g + 1.0) * c) * (uk - ss)
        uf = 2.0 / (g + 1.0) * (c + 0.5 * (g - 1.0) * uk + ss)
        return rho * base ** (2.0 / (g - 1.0)), sign * -uf, pk * base ** (2.0 * g / (g - 1.0))

    def sample(svec):
        out = np.array([state(s, left, -1.0) if s <= u else state(s, right, 1.0) for s in svec])
        return out[:, 0], out[:, 1], out[:, 2]

    return p, u, sample


def test_exact_riemann_matches_toro_sod():
    """The exact solver on Toro's Sod problem (his Table 4.3: p* = 0.30313, u* = 0.92745), as the
    reference's verify.py checks its own before trusting it."""
    p, u, sample = exact_riemann((1.0, 0.0, 1.0), (0.125, 0.0, 0.1), 1.4)
    assert abs(p - 0.30313) <= 1e-5 and abs(u - 0.92745) <= 1e-5
    rho, uu, pp = sample(np.array([-2.0, -0.5, 0.0, 0.9, 1.5, 2.0]))
    assert rho[0] == 1.0 and pp[0] == 1.0 and rho[-1] == 0.125 and pp[-1] == 0.1
    assert abs(uu[3] - u) <= 1e-12 and abs(pp[3] - p) <= 1e-12 and abs(pp[4] - p) <= 1e-12


def _sod_checks(lib):
    """An anisotropic Sod tube (P11 left 1e5, right 1e4; P22 = P33 = 0.01 rho), explicit Euler, first
    order, CFL 0.8, 400 x 4 cells with walls on the j faces: in 1-D the AG system is the gamma = 3 Euler
    system in (rho, rho u, rho u^2 + P11). Gates of the reference's verify.py: finite, min P11 above 1e3,
    L1(rho) within 0.05, P22/rho passive to 1e-9, total variation of rho and P11 within 1.05 times the
    exact one."""
    g = {k[4:]: float(GOLD[k]) for k in GOLD.files if k.startswith("sod_")}
    nx, ny = int(g["NX"]), int(g["NY"])
    xc = (np.arange(nx) + 0.5) * g["LX"] / nx
    left = xc < g["X0"]
    rho = np.where(left, g["RHO_L"], g["RHO_R"])
    zero = np.zeros(nx)
    ic = np.stack([rho, zero, zero, zero, np.where(left, g["P_L"], g["P_R"]), zero, zero, g["PT_RATIO"] * rho,
                   zero, g["PT_RATIO"] * rho, zero + g["T0"], rho / (4.0 / 3.0 * math.pi * g["RP"] ** 3 * g["RHO_M"])])
    case = configs.ag_tube(ic, x0=0.0, lx=g["LX"], ny=ny, ly=g["LY"], h=g["H"], side_code=300, scheme="euler",
                           limiter="IORD", cfl=0.8, dt_max=1e-3, t_end=g["t"], rho_al=g["RHO_M"], cs=1000.0)
    t, p = _run(case, lib, g["t"])
    assert t >= g["T_END"] * (1.0 - 1e-12)
    assert np.isfinite(p).all()
    rho_n, p11, p22 = p[..., 0], p[..., 4], p[..., 7]
    _, _, sample = exact_riemann((g["RHO_L"], 0.0, g["P_L"]), (g["RHO_R"], 0.0, g["P_R"]), g["GAMMA"])
    rho_ex, _, p_ex = sample((xc - g["X0"]) / t)
    l1 = float(np.abs(rho_n.mean(axis=0) - rho_ex).sum() / rho_ex.sum())
    tv = lambda a: float(np.abs(np.diff(a)).sum())
    assert float(p11.min()) > g["P11_MIN"]
    assert l1 <= g["L1_TOL"], l1
    assert float(np.abs(p22 / rho_n - g["PT_RATIO"]).max()) < g["PT_TOL"]
    assert tv(rho_n.mean(axis=0)) / tv(rho_ex) <= g["TV_TOL"]
    assert tv(p11.mean(axis=0)) / tv(p_ex) <= g["TV_TOL"]
    return l1


BERTHON = ("SCS", "RCS", "RCR", "SCS-hlle")


@pytest.mark.parametrize("name", BERTHON)
def test_berthon_oracle(orc, name):
    _berthon_checks(orc, name)


def test_sod_ag_oracle(orc):
    _sod_checks(orc)


@pytest.mark.gpu
@pytest.mark.parametrize("name", BERTHON)
def test_berthon_gpu(name):
    _berthon_checks(_gpu(), name)


@pytest.mark.gpu
def test_sod_ag_gpu():
    _sod_checks(_gpu())
