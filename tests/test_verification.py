"""The reference's drag- and thermal-relaxation verification cases (test/verification/A-drag-relaxation,
B-thermal-relaxation, C-advection-sine, D-drag-matrix, E-heat-matrix, F-evaporation parts 1-4,
G-cloud-translation, H-linear-strain, I-vortex-cloud, J-tau-limit, L-materials legs 1 and 2) on the oracle and on the CUDA path (plain FP64 form). A: a uniform MK cloud at rest in a uniform gas stream under
Stokes drag relaxes as u_g + (u_p0 - u_g) exp(-t/tau), tau = rho_al dp^2 / (18 mu). The gates are the
reference's: the velocity within 1e-5 of u_g at t/tau = 0.1 ... 5, the field uniform to 1e-12 u_g,
density unchanged to 1e-12, number density to 1e-9, temperature to 1e-9 T_g; and observed orders of
the time integration within 0.35 of 2 (RK2) and 3 (RK3) when the CFL number halves. B: a cloud moving
with the gas at 400 K in a 300 K gas relaxes as T_g + (T_p0 - T_g) exp(-t/tau_T), tau_T = rho_al cs
dp^2 / (12 k), within 1e-5 of the initial gap; uniform to 1e-10 T_p0; velocity, density and number
density unchanged."""
import cmath
import math

import numpy as np
import pytest

from ice_b200 import abi, configs
from ice_b200.solver import Solver

TAU = 1000.0 * 1e-4 ** 2 / (18.0 * 1.8e-5)
UG, TG = 10.0, 300.0


def _gpu():
    from ice_b200 import build
    build.build()
    return abi.load_gpu()


def _relaxation_checks(lib):
    for ratio in (0.1, 0.5, 1.0, 2.0, 3.0, 5.0):
        n = int(math.ceil(ratio * TAU / 1e-4 - 1e-9))        # dt-max (1e-4 s) sets the step here
        s = Solver(configs.relaxation_tube(steps=n), lib)
        out = s.step(n)
        assert out.status == 0 and out.dtglobal == 1e-4
        p = s.download(0, 0)[2, 2, 2:-2]
        exact = UG + (0.0 - UG) * math.exp(-out.time / TAU)
        u = p[:, 1]
        assert abs(u[0] - exact) <= 1e-5 * UG
        assert u.max() - u.min() <= 1e-12 * UG
        assert np.all(np.abs(p[:, 0] - 1.0) <= 1e-12)
        assert np.all(np.abs(p[:, 5] / p[0, 5] - 1.0) <= 1e-9)
        assert np.all(np.abs(p[:, 4] - TG) <= 1e-9 * TG)


def _order_checks(lib):
    for rk, expected in (("RK2", 2.0), ("RK3", 3.0)):
        errors = []
        for cfl in (0.8, 0.4, 0.2):
            s = Solver(configs.relaxation_tube(nx=10, ny=2, lx=0.01, ly=1e-2, scheme=rk, cfl=cfl, vg=50.0), lib)
            t = 0.0
            while t < 0.02 - 1e-15:
                t = s.step(1).time
            u = s.download(0, 0)[2, 2, 2, 1]
            errors.append(abs(u - (UG - UG * math.exp(-t / TAU))) / UG)
        orders = [math.log(errors[i] / errors[i + 1]) / math.log(2.0) for i in range(2)]
        usable = [o for o, e in zip(orders, errors[1:]) if e > 1e-12]
        assert usable and min(usable) >= expected - 0.35, (rk, errors, orders)


def _thermal_checks(lib):
    tau_t = 1000.0 * 900.0 * 1e-4 ** 2 / (12.0 * 0.026)
    for ratio in (0.1, 0.5, 1.0, 2.0, 3.0, 5.0):
        n = int(math.ceil(ratio * tau_t / 1e-4 - 1e-9))
        s = Solver(configs.relaxation_tube(steps=n, up0=UG, tp0=400.0), lib)
        out = s.step(n)
        assert out.status == 0
        p = s.download(0, 0)[2, 2, 2:-2]
        exact = TG + (400.0 - TG) * math.exp(-out.time / tau_t)
        temp = p[:, 4]
        assert abs(temp[0] - exact) <= 1e-5 * (400.0 - TG)
        assert temp.max() - temp.min() <= 1e-10 * 400.0
        assert np.all(np.abs(p[:, 1] - UG) <= 1e-12 * UG)
        assert np.all(np.abs(p[:, 0] - 1.0) <= 1e-12)
        assert np.all(np.abs(p[:, 5] / p[0, 5] - 1.0) <= 1e-9)


DRAG_LAWS = ("Newton", "Stokes", "Schlichting", "Schiller-Naumann", "Wen-Yu", "Putnam", "Clift-Gauvin",
             "Morsi-Alexander", "Carlson-Hoglund", "Henderson", "Crowe", "Hermsen")
STOKES_LIMIT = ("Stokes", "Schlichting", "Schiller-Naumann", "Wen-Yu", "Putnam", "Clift-Gauvin", "Morsi-Alexander")
COMPRESSIBLE = ("Carlson-Hoglund", "Henderson", "Crowe", "Hermsen")


def _rk4_reference(orc, law, ug, t_end, steps=5000):
    """du/dt = (u_g - u)/tau(u) with the solver's relaxation time 8 rho_al r_p / (3 rho_g Cd |slip| + 1e-20)
    and Cd of the law (the oracle's correlation, itself pinned against the reference's), by classic RK4
    with u(0) = 0 and the particles at the gas temperature."""
    rho_g, mu, rp, rho_al = 1.2, 1.8e-5, 0.5e-4, 1000.0
    sound = math.sqrt(1.4 * 287.05 * TG)
    sel = abi.DRAG[law]

    def rhs(u):
        slip = ug - u
        re = 2.0 * rho_g * rp * abs(slip) / mu
        cd = orc.drag(re, abs(slip) / sound, 1.4, 1.0, sel)
        return slip / (8.0 * rho_al * rp / (3.0 * rho_g * cd * abs(slip) + 1.0e-20))
    h, u = t_end / steps, 0.0
    for _ in range(steps):
        k1 = rhs(u); k2 = rhs(u + 0.5 * h * k1); k3 = rhs(u + 0.5 * h * k2); k4 = rhs(u + h * k3)
        u += h / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4)
    return u


def _drag_run(lib, law, ug, t_end, **mesh):
    s = Solver(configs.relaxation_tube(drag=law, ug=ug, vg=mesh.pop("vg", 0.0), **mesh), lib)
    t = 0.0
    while t < t_end - 1e-15:
        out = s.step(1)
        assert out.status == 0
        t = out.time
    p = s.download(0, 0)[2, 2:-2, 2:-2]
    return t, p


def _drag_matrix_checks(lib, orc):
    # vanishing slip: the laws built as Stokes times a correction tend to the Stokes exponential
    for law in STOKES_LIMIT:
        t, p = _drag_run(lib, law, 1e-3, 0.03)
        assert abs(p[0, 0, 1] - 1e-3 * (1.0 - math.exp(-t / TAU))) <= 0.01 * 1e-3, law
    # Re = 67: every law against the integration of its own relaxation time; the temperature stays
    for law in DRAG_LAWS:
        t, p = _drag_run(lib, law, UG, 0.03)
        assert abs(p[0, 0, 1] - _rk4_reference(orc, law, UG, t)) <= 1e-3 * UG, law
        assert np.all(np.abs(p[..., 4] - TG) <= 1e-9 * TG), law
    # above Re = 1000 (the branched laws switch formula), and transonic and supersonic slip (the
    # compressible laws' branches), with a transverse velocity shared with the gas keeping dt short
    for ug, laws, t_end in ((200.0, DRAG_LAWS, 4e-3), (450.0, COMPRESSIBLE, 2e-3), (900.0, COMPRESSIBLE, 2e-3)):
        for law in laws:
            t, p = _drag_run(lib, law, ug, t_end, vg=ug, lx=0.01, ly=2.5e-3, lz=1.25e-3, ny=2)
            assert abs(p[0, 0, 1] - _rk4_reference(orc, law, ug, t)) <= 1e-3 * ug, (law, ug)


HEAT_LAWS = ("Stokes", "JAXA1", "JAXA2", "JAXA3", "JAXA4", "Ranz-Marshall", "Kavanau-Drake")
NU2_LIMIT = ("Stokes", "JAXA2", "JAXA3", "Ranz-Marshall")
KG, CS, MU = 0.026, 900.0, 1.8e-5
PR = 1.4 / 0.4 * 287.05 * MU / KG


def _heat_rk4(orc, law, ug, t_end, tp0=400.0, steps=5000):
    """du/dt = (u_g - u)/tau_Stokes and dT/dt = 2 Nu kg pi r_p n (T_g - T)/(rho_p cs), Nu of the law (the
    oracle's correlation, pinned against the reference's) at the slip's Re and Ma, by classic RK4."""
    rho_g, rp, rho_p = 1.2, 0.5e-4, 1.0
    n = rho_p / (1000.0 * 4.0 / 3.0 * math.pi * rp ** 3)
    sound = math.sqrt(1.4 * 287.05 * TG)
    sel = abi.HEAT[law]

    def rhs(u, T):
        slip = ug - u
        re = 2.0 * rho_g * rp * abs(slip) / MU
        nu = orc.heat(re, PR, abs(slip) / sound, sel)
        return slip / TAU, 2.0 * nu * KG * math.pi * rp * n * (TG - T) / (rho_p * CS)
    h, u, T = t_end / steps, 0.0, tp0
    for _ in range(steps):
        k1 = rhs(u, T)
        k2 = rhs(u + 0.5 * h * k1[0], T + 0.5 * h * k1[1])
        k3 = rhs(u + 0.5 * h * k2[0], T + 0.5 * h * k2[1])
        k4 = rhs(u + h * k3[0], T + h * k3[1])
        u += h / 6.0 * (k1[0] + 2 * k2[0] + 2 * k3[0] + k4[0])
        T += h / 6.0 * (k1[1] + 2 * k2[1] + 2 * k3[1] + k4[1])
    return u, T


def _heat_matrix_checks(lib, orc):
    tau_t = 1000.0 * CS * 1e-4 ** 2 / (12.0 * KG)
    # vanishing slip: the laws with Nu -> 2 follow the exact Nu = 2 relaxation
    for law in NU2_LIMIT:
        s = Solver(configs.relaxation_tube(heat=law, ug=1e-3, tp0=400.0, steps=300), lib)
        out = s.step(300)
        T = s.download(0, 0)[2, 2, 2, 4]
        assert abs(T - (TG + 100.0 * math.exp(-out.time / tau_t))) <= 0.05 * 100.0, law
    # Re = 67: temperature and velocity against the RK4 integration of the coupled pair
    for law in HEAT_LAWS:
        s = Solver(configs.relaxation_tube(heat=law, tp0=400.0, steps=300), lib)
        out = s.step(300)
        p = s.download(0, 0)[2, 2, 2:-2]
        uref, tref = _heat_rk4(orc, law, UG, out.time)
        assert abs(p[0, 4] - tref) <= 1e-3 * 100.0, law
        assert abs(p[0, 1] - uref) <= 1e-3 * UG, law
        assert p[:, 4].max() - p[:, 4].min() <= 1e-10 * 400.0, law
    # constant slip (no drag): JAXA4's Nu is frozen and the cooling an exact exponential
    sound = math.sqrt(1.4 * 287.05 * TG)
    re = 2.0 * 1.2 * 0.5e-4 * UG / MU
    tau_j = tau_t * 2.0 / orc.heat(re, PR, UG / sound, abi.HEAT["JAXA4"])
    s = Solver(configs.relaxation_tube(heat="JAXA4", drag="NoDrag", tp0=400.0, steps=100), lib)
    out = s.step(100)
    p = s.download(0, 0)[2, 2, 2:-2]
    assert abs(p[0, 4] - (TG + 100.0 * math.exp(-out.time / tau_j))) <= 3e-4 * 100.0
    assert np.all(p[:, 1] == 0.0)


def _tau_limit_checks(lib):
    """J1: drops of 2 um (tau_p = 2.2e-5 s = dt-max / 4.5) at rest in a 10 m/s stream, SSP-RK3. The first
    step cannot know tau and takes dt-max; every later step is tau_p, so (t - dt-max)/tau_p is an
    integer, and the cloud relaxes. J1a: tau-factor 0.2 and dt-max 5e-6 follow the exponential."""
    kw = dict(dp=2e-6, rho_al=2000.0, cs=1000.0, rho_g=1.0, mu=2e-5, kg=0.025, scheme="RK3", cfl=0.8)
    tau = 2000.0 * 2e-6 ** 2 / (18.0 * 2e-5)
    for tf, dt_max, t_end, gate in ((1.0, 1e-4, 20.0 * tau, None), (0.2, 5e-6, 2.0 * tau, 5e-3)):
        s = Solver(configs.relaxation_tube(tau_factor=tf, dt_max=dt_max, **kw), lib)
        t = s.step(1).time
        if tf == 1.0:       # the first step, dt-max = 4.5 tau: SSP-RK3's R(-4.5) = -8.5625, u_p = 95.625
            assert abs(s.download(0, 0)[2, 2, 2, 1] - 95.625) <= 1e-10 * 95.625
        while t < t_end - 1e-15:
            out = s.step(1)
            assert out.status == 0
            t = out.time
        u = s.download(0, 0)[2, 2, 2:-2, 1]
        k = (t - dt_max) / (tf * tau)
        assert k >= 1.0 and abs(k - round(k)) <= 1e-6, (tf, k)
        if gate is None:
            assert np.all(np.abs(u / UG - 1.0) < 1e-3)
        else:
            assert np.all(np.abs(u - UG * (1.0 - math.exp(-t / tau))) / UG < gate)


def _advection_checks(lib):
    """C: a sine density wave carried at 1 m/s around a periodic slab for 0.25 s at dt = 1e-4 on 25-200
    cells: mass conserved to 1e-12, velocity uniform to 1e-10, the L1 error against the shifted exact
    cell averages converging at order >= 1.5 (MUSCL, van Leer) and >= 0.85 (first order), MUSCL the more
    accurate on every grid."""
    k = 2.0 * math.pi

    def avg(xl, xr, t):
        return 10.0 + 5.0 * (math.cos(k * (xl - t)) - math.cos(k * (xr - t))) / (k * (xr - xl))
    grids = (25, 50, 100, 200)
    res = {}
    for lim, expected in (("vanleer", 1.5), ("IORD", 0.85)):
        errors = []
        for nx in grids:
            s = Solver(configs.periodic_sine(nx, lim), lib)
            out = s.step(2500)
            assert out.status == 0 and out.dtglobal == 1e-4
            p = s.download(0, 0)[2, 2, 2:-2]
            dx = 1.0 / nx
            ref = np.array([avg(i * dx, (i + 1) * dx, out.time) for i in range(nx)])
            errors.append(float(np.sum(np.abs(p[:, 0] - ref))) / nx / 5.0)
            m0 = sum(avg(i * dx, (i + 1) * dx, 0.0) for i in range(nx)) * dx
            assert abs(float(np.sum(p[:, 0])) * dx - m0) <= 1e-12 * m0
            assert np.all(np.abs(p[:, 1] - 1.0) <= 1e-10)
        orders = [math.log(errors[i] / errors[i + 1]) / math.log(2.0) for i in range(len(grids) - 1)]
        assert min(orders) >= expected, (lim, errors, orders)
        res[lim] = errors
    assert all(a < b for a, b in zip(res["vanleer"], res["IORD"]))


def _evaporation_checks(lib):
    """F, parts 1-4 (part 1: at frozen droplet temperature every evaporation model follows the d-squared law; its
    slope K against the one the reference computes from the published correlations
    (tests/golden/evaporation.npz) to 1e-6; the field uniform, the number density unchanged, the
    temperature held to 1e-3 K. CEM with the Langmuir-Knudsen interface against the reference's RK4
    integration, bulk density to 1e-8. Evaporation off: the bulk density untouched to 1e-14. Parts 2-4
    below.)"""
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / "evaporation.npz")
    n0 = 1.0 / (4.0 / 3.0 * math.pi * 0.5e-4 ** 3 * 1000.0)
    diameter = lambda r: 2.0 * (0.75 * r / (n0 * math.pi * 1000.0)) ** (1.0 / 3.0)
    for model, k_ref in zip(g["models"], g["K"]):
        s = Solver(configs.evaporating_tube(str(model)), lib)
        out = s.step(2000)
        assert out.status == 0
        p = s.download(0, 0)[2, 2, 2:-2]
        k_ice = (1e-4 ** 2 - diameter(p[0, 0]) ** 2) / out.time
        assert abs(k_ice - k_ref) <= 1e-6 * k_ref, (model, k_ice, k_ref)
        assert p[:, 0].max() - p[:, 0].min() <= 1e-12
        assert np.all(np.abs(p[:, 5] - n0) <= 1e-9 * n0)
        assert np.all(np.abs(p[:, 4] - 300.0) <= 1e-3)
    s = Solver(configs.evaporating_tube("CEM", "LK"), lib)
    s.step(2000)
    assert abs(s.download(0, 0)[2, 2, 2, 0] - float(g["rho_lk"])) <= 1e-8
    s = Solver(configs.evaporating_tube("none"), lib)
    s.step(2000)
    assert abs(s.download(0, 0)[2, 2, 2, 0] - 1.0) <= 1e-14
    # part 2: the temperature released (cp 4180, 0.05 s at dt-max 5e-6) against the reference's RK4 of
    # the coupled (rho_p, T_p) system: T_p to 1e-8 of the initial gap, rho_p to 1e-9
    for model, (rho_ref, t_ref) in zip(g["free"], g["hot"]):
        s = Solver(configs.evaporating_tube(str(model), cs=4180.0, dt_max=5e-6, steps=10000), lib)
        s.step(10000)
        p = s.download(0, 0)[2, 2, 2]
        assert abs(p[4] - t_ref) <= 1e-8 * 500.0 and abs(p[0] - rho_ref) <= 1e-9, model
    assert g["hot"][0][1] - 300.0 > 1.0                  # without blowing the d2-law droplet heats up
    # part 3: d2-law with Nu = 2 and the blowing correction is exactly isothermal, on the d-squared law
    s = Solver(configs.evaporating_tube("d2-law", cs=4180.0, dt_max=5e-6, steps=10000, blowing=True), lib)
    out = s.step(10000)
    p = s.download(0, 0)[2, 2, 2:-2]
    assert np.all(np.abs(p[:, 4] - 300.0) <= 1e-8)
    k_ice = (1e-4 ** 2 - diameter(p[0, 0]) ** 2) / out.time
    assert abs(k_ice - g["K"][0]) <= 1e-6 * g["K"][0]
    # part 4: above the boiling point (380 K) on the boiling clamp, each model's slope to 1e-5 and CEM
    # with the Langmuir-Knudsen interface to 1e-8, over the time CEM takes to lose 10 % of its mass
    t_boil = float(g["t_boil"])
    for model, k_ref in zip(g["models"], g["K_boil"]):
        s = Solver(configs.evaporating_tube(str(model), dt_max=t_boil / 1000.0, steps=1000, tp0=380.0), lib)
        out = s.step(1000)
        assert out.status == 0
        k_ice = (1e-4 ** 2 - diameter(s.download(0, 0)[2, 2, 2, 0]) ** 2) / out.time
        assert abs(k_ice - k_ref) <= 1e-5 * k_ref, model
    s = Solver(configs.evaporating_tube("CEM", "LK", dt_max=t_boil / 1000.0, steps=1000, tp0=380.0), lib)
    s.step(1000)
    assert abs(s.download(0, 0)[2, 2, 2, 0] - float(g["rho_lk_boil"])) <= 1e-8


def _translation_checks(lib):
    """G: a cloud at rest released into a uniform 10 m/s gas on a periodic slab translates rigidly while
    its drops relax. Every run: the density-weighted particle velocity within 1e-6 of the exact
    relaxation, mass to 1e-12, the centroid within 0.05 cells of the exact displacement. A smooth
    (Gaussian) cloud converges in space at order >= 1.5 (50-200 cells); the spread of u_p vanishes at
    order >= 1.8 in dt and is below 1e-6 at dt 5e-6; a top hat keeps mass and centroid."""
    tau = TAU
    t_end = 3.0 * tau

    def avg(shape, xl, xr, shift, m=32):
        h = (xr - xl) / m
        return float(np.mean(configs.cloud_profile(shape, (xl + (np.arange(m) + 0.5) * h - shift) % 1.0)))

    def run(nx, shape, dt):
        n = int(math.ceil(t_end / dt - 1e-9))
        s = Solver(configs.periodic_cloud(nx, shape, dt, n), lib)
        out = s.step(n)
        assert out.status == 0
        return out.time, s.download(0, 0)[2, 2, 2:-2]

    def common(t, p, shape, nx):
        dx = 1.0 / nx
        rho, up = p[:, 0], p[:, 1]
        assert abs(float(np.sum(rho * up) / np.sum(rho)) - UG * (1.0 - math.exp(-t / tau))) <= 1e-6 * UG
        m0 = sum(avg(shape, i * dx, (i + 1) * dx, 0.0) for i in range(nx)) * dx
        assert abs(float(rho.sum()) * dx / m0 - 1.0) <= 1e-12
        x = UG * t - UG * tau * (1.0 - math.exp(-t / tau))
        ang = np.sum(rho * np.exp(2j * np.pi * (np.arange(nx) + 0.5) * dx))
        drift = abs((math.atan2(ang.imag, ang.real) / (2.0 * math.pi)) % 1.0 - (0.25 + x) % 1.0)
        assert min(drift, 1.0 - drift) <= 0.05 * dx
        return x

    errors = []
    for nx in (50, 100, 200):
        t, p = run(nx, "gauss", 1e-5)
        x = common(t, p, "gauss", nx)
        dx = 1.0 / nx
        ref = np.array([avg("gauss", i * dx, (i + 1) * dx, x) for i in range(nx)])
        errors.append(float(np.abs(p[:, 0] - ref).sum() / ref.sum()))
    assert min(math.log(errors[i] / errors[i + 1]) / math.log(2.0) for i in range(2)) >= 1.5, errors
    spreads = []
    for dt in (2e-5, 1e-5, 5e-6):
        _, p = run(100, "gauss", dt)
        spreads.append(float(p[:, 1].max() - p[:, 1].min()) / UG)
    assert min(math.log(spreads[i] / spreads[i + 1]) / math.log(2.0) for i in range(2)) >= 1.8, spreads
    assert spreads[-1] <= 1e-6
    t, p = run(100, "tophat", 1e-5)
    common(t, p, "tophat", 100)


def _strain_checks(lib):
    """H: a Gaussian cloud seeded at the local velocity of a frozen gas in the uniform strain
    u_g = 2 + 6 x. With xi = x + 1/3 every drop is displaced by one factor C(t) (C'' tau + C' = 6 C,
    C(0) = 1, C'(0) = 6), so rho_p = rho_p0(xi / C - 1/3) / C and u_p = (C'/C) xi exactly. At St = 0.185,
    on 100-400 cells: centroid within 0.05 cells, the density-weighted slope of u_p against xi within
    2e-4 of C'/C, mass within 2e-3 of the exact stretch, L1 order >= 1.5. Over St = 0.2 to 0.025 on 200
    cells the slip coefficient 6 - slope tends to the asymptote 36 tau monotonically, departs from it by
    1.3-2.2 St, and is within 5 % of it at St = 0.025."""
    def stretch(tau, t, a=6.0):
        root = math.sqrt(1.0 + 4.0 * a * tau)
        lp, lm = (-1.0 + root) / (2.0 * tau), (-1.0 - root) / (2.0 * tau)
        ca, cb = (a - lm) / (lp - lm), (lp - a) / (lp - lm)
        return (ca * math.exp(lp * t) + cb * math.exp(lm * t),
                ca * lp * math.exp(lp * t) + cb * lm * math.exp(lm * t))

    def profile(x):
        return 10.0 * (np.exp(-(x - 0.2) ** 2 / (2.0 * 0.035 ** 2)) + 1e-6)

    def run(nx, tau):
        n = int(math.ceil(0.1 / 2e-5 - 1e-9))
        s = Solver(configs.strain_tube(nx, math.sqrt(18.0 * 1.8e-5 * tau / 1000.0), n), lib)
        out = s.step(n)
        assert out.status == 0
        p = s.download(0, 0)[2, 2, 2:-2]
        xi = (np.arange(nx) + 0.5) / nx + 1.0 / 3.0
        slope = float(np.sum(p[:, 0] * p[:, 1] * xi) / np.sum(p[:, 0] * xi ** 2))
        return out.time, p, xi, slope

    errors = []
    for nx in (100, 200, 400):
        t, p, xi, slope = run(nx, TAU)
        c, cdot = stretch(TAU, t)
        dx = 1.0 / nx
        sub = np.arange(nx)[:, None] * dx + (np.arange(32)[None, :] + 0.5) * (dx / 32) + 1.0 / 3.0
        ref = (profile(sub / c - 1.0 / 3.0) / c).mean(axis=1)
        rho = p[:, 0]
        errors.append(float(np.abs(rho - ref).sum() / ref.sum()))
        xbar = float(np.sum(rho * xi) / rho.sum())
        assert abs(xbar - c * (0.2 + 1.0 / 3.0)) <= 0.05 * dx
        assert abs(slope / (cdot / c) - 1.0) <= 2e-4
        assert abs(float(rho.sum() / ref.sum()) - 1.0) <= 2e-3
    assert min(math.log(errors[i] / errors[i + 1]) / math.log(2.0) for i in range(2)) >= 1.5, errors
    stokes, ratios = (0.2, 0.1, 0.05, 0.025), []
    for st in stokes:
        tau = st / 6.0
        t, p, xi, slope = run(200, tau)
        c, cdot = stretch(tau, t)
        assert abs(slope / (cdot / c) - 1.0) <= 5e-4
        ratios.append((6.0 - slope) / (36.0 * tau))
    assert all(a < b for a, b in zip(ratios[:-1], ratios[1:])), ratios
    assert all(1.3 * st <= 1.0 - r <= 2.2 * st for r, st in zip(ratios, stokes)), ratios
    assert abs(ratios[-1] - 1.0) <= 0.05


def _vortex_checks(lib):
    """I: a Gaussian cloud seeded at the local velocity of a frozen gas in solid-body rotation
    (Omega = 1) on [-2, 2]^2, a quarter turn. In z = x + i y every drop is displaced by one complex
    factor C(t), so rho_p = rho_p0(z / C) / |C|^2 and u_p + i v_p = (C'/C) z. At St = 0.1 on 48-192
    cells a side: centroid within 0.1 cells of C z_0, L1 and centroid orders >= 1.5. Over St = 0.01 to 10
    on 96 cells: radius within 5e-3 and phase lag within 5e-3 rad of C, the velocity slope within 1e-2
    of C'/C, L1 <= 0.15, mass within 1e-3; lag and radius grow with St, St = 0.01 is a tracer (lag
    <= 5e-3, radius within 0.02) and St = 10 lags at least 0.4 rad."""
    quarter = 0.5 * math.pi

    def stretch(tau, t):
        root = cmath.sqrt(1.0 + 4.0j * tau)
        lp, lm = (-1.0 + root) / (2.0 * tau), (-1.0 - root) / (2.0 * tau)
        ca, cb = (1.0j - lm) / (lp - lm), (lp - 1.0j) / (lp - lm)
        return (ca * cmath.exp(lp * t) + cb * cmath.exp(lm * t),
                ca * lp * cmath.exp(lp * t) + cb * lm * cmath.exp(lm * t))

    def run(n, tau):
        steps = int(math.ceil(quarter / 1e-3 - 1e-9))
        s = Solver(configs.vortex_box(n, tau, steps), lib)
        out = s.step(steps)
        assert out.status == 0
        p = s.download(0, 0)[2, 2:-2, 2:-2]
        c = -2.0 + (np.arange(n) + 0.5) * (4.0 / n)
        y, x = np.meshgrid(c, c, indexing="ij")
        z = x + 1j * y
        rho, w = p[..., 0], p[..., 1] + 1j * p[..., 2]
        c_t, cdot = stretch(tau, out.time)
        z0 = z / c_t
        ref = 10.0 * (np.exp(-((z0.real - 0.6) ** 2 + z0.imag ** 2) / (2.0 * 0.12 ** 2)) + 1e-8) / abs(c_t) ** 2
        centre = complex(np.sum(rho * z) / rho.sum())
        slope = complex(np.sum(rho * w * z.conj()) / np.sum(rho * abs(z) ** 2))
        err = float(np.abs(rho - ref).sum() / ref.sum())
        return out.time, c_t, cdot, centre, slope, err, float(rho.sum() / ref.sum())

    errors, drifts = [], []
    for n in (48, 96, 192):
        _, c_t, _, centre, _, err, _ = run(n, 0.1)
        errors.append(err)
        drifts.append(abs(centre - 0.6 * c_t))
        assert drifts[-1] <= 0.1 * 4.0 / n
    for e in (errors, drifts):
        assert min(math.log(e[i] / e[i + 1]) / math.log(2.0) for i in range(2)) >= 1.5, e
    lags, radii = [], []
    for st in (0.01, 0.1, 1.0, 10.0):
        t, c_t, cdot, centre, slope, err, mass = run(96, st)
        lags.append(t - cmath.phase(centre))
        radii.append(abs(centre) / 0.6)
        assert abs(radii[-1] / abs(c_t) - 1.0) <= 5e-3
        assert abs(lags[-1] - (t - cmath.phase(c_t))) <= 5e-3
        assert abs(slope / (cdot / c_t) - 1.0) <= 1e-2
        assert err <= 0.15
        assert abs(mass - 1.0) <= 1e-3
    assert all(a < b for a, b in zip(lags[:-1], lags[1:])), lags
    assert all(a < b for a, b in zip(radii[:-1], radii[1:])), radii
    assert lags[0] <= 5e-3 and abs(radii[0] - 1.0) <= 0.02
    assert lags[-1] >= 0.4


def _materials_checks(lib):
    """L, legs 1 and 2: several MK families in one case, each on its own material. L1: two families
    with the same state (2 kg/m3, 1e-4 m drops of density 2000) at rest at 300 K in a gas at rest at
    400 K, NoDrag, heat Stokes; materials A (cp 1000, density 2000) and B (cp 2000, density 1000); each
    relaxes with its own tau = rho_p cp / (4 pi k R_p n), R_p from the state and its own density, to
    1e-6 of the gap at t = tau_A (dt-max = tau_A / 1000); L1b: families 1 and 2 on A, 3 on B. L2: case F's
    frozen cloud, family A evaporating (CEM) on the d-squared slope of the reference's correlations to
    1e-6, family B (evaporation off, cp 2000, density 2000) keeps its bulk and number densities to the
    last bit."""
    from pathlib import Path
    rho_p = 1e-3 * 2000.0
    n = rho_p / (2000.0 * 4.0 / 3.0 * math.pi * 0.5e-4 ** 3)
    mats = {"A": (1000.0, 2000.0), "B": (2000.0, 1000.0)}

    def tau(m):
        cp, rho_m = mats[m]
        rp = (0.75 * rho_p / (n * math.pi * rho_m)) ** (1.0 / 3.0)
        return rho_p * cp / (4.0 * math.pi * 0.026 * rp * n)

    for fam_mat in (("A", "B"), ("A", "A", "B")):
        t_end, dt = tau("A"), min(tau("A"), tau("B")) / 1000.0
        steps = int(math.ceil(t_end / dt - 1e-9))
        case = configs.relaxation_tube(dt_max=dt, steps=steps, drag="NoDrag", heat="Stokes", ug=0.0,
                                       rho_al=2000.0, cs=1000.0)
        case.gas = [configs._gas_layout(case, 0, 1.2, 0.0, 0.0, 0.0, 400.0)]
        configs.with_families(case, [configs.Family("MK", rho_al=mats[m][1], cs_al=mats[m][0]) for m in fam_mat])
        s = Solver(case, lib)
        out = s.step(steps)
        assert out.status == 0 and out.time >= t_end * (1.0 - 1e-12)
        for q, m in enumerate(fam_mat):
            temp = s.download(0, q)[2, 2, 2:-2, 4]
            ref = 400.0 - 100.0 * math.exp(-out.time / tau(m))
            assert float(np.abs(temp - ref).max()) / 100.0 <= 1e-6, (fam_mat, q, m)
    g = np.load(Path(__file__).resolve().parent / "golden" / "evaporation.npz")
    k_ref = float(g["K"][list(g["models"]).index("CEM")])
    case = configs.evaporating_tube("CEM")
    b = configs.Family("MK", rho_al=2000.0, cs_al=2000.0, lv_al=2.26e6, evap="none", Mv=18.015, Tboil=373.15)
    configs.with_families(case, [case.families[0], b])
    s = Solver(case, lib)
    out = s.step(2000)
    assert out.status == 0
    n0 = 1.0 / (4.0 / 3.0 * math.pi * 0.5e-4 ** 3 * 1000.0)
    pa, pb = s.download(0, 0)[2, 2, 2:-2], s.download(0, 1)[2, 2, 2:-2]
    k_ice = (1e-4 ** 2 - (2.0 * (0.75 * pa[0, 0] / (n0 * math.pi * 1000.0)) ** (1.0 / 3.0)) ** 2) / out.time
    assert abs(k_ice - k_ref) <= 1e-6 * k_ref
    assert pa[:, 0].max() - pa[:, 0].min() <= 1e-12
    assert np.all(pb[:, 0] == 1.0) and np.all(pb[:, 5] == n0)


def test_drag_relaxation_oracle(orc):
    _relaxation_checks(orc)
    _order_checks(orc)


def test_thermal_relaxation_oracle(orc):
    _thermal_checks(orc)


def test_drag_matrix_oracle(orc):
    _drag_matrix_checks(orc, orc)


def test_heat_matrix_oracle(orc):
    _heat_matrix_checks(orc, orc)


def test_tau_limit_oracle(orc):
    _tau_limit_checks(orc)


def test_advection_oracle(orc):
    _advection_checks(orc)


def test_evaporation_oracle(orc):
    _evaporation_checks(orc)


def test_translation_oracle(orc):
    _translation_checks(orc)


def test_strain_oracle(orc):
    _strain_checks(orc)


def test_vortex_oracle(orc):
    _vortex_checks(orc)


def test_materials_oracle(orc):
    _materials_checks(orc)


@pytest.mark.gpu
def test_drag_relaxation_gpu():
    gpu = _gpu()
    _relaxation_checks(gpu)
    _order_checks(gpu)


@pytest.mark.gpu
def test_thermal_relaxation_gpu():
    _thermal_checks(_gpu())


@pytest.mark.gpu
def test_drag_matrix_gpu(orc):
    _drag_matrix_checks(_gpu(), orc)


@pytest.mark.gpu
def test_heat_matrix_gpu(orc):
    _heat_matrix_checks(_gpu(), orc)


@pytest.mark.gpu
def test_tau_limit_gpu():
    _tau_limit_checks(_gpu())


@pytest.mark.gpu
def test_advection_gpu():
    _advection_checks(_gpu())


@pytest.mark.gpu
def test_evaporation_gpu():
    _evaporation_checks(_gpu())


@pytest.mark.gpu
def test_translation_gpu():
    _translation_checks(_gpu())


@pytest.mark.gpu
def test_strain_gpu():
    _strain_checks(_gpu())


@pytest.mark.gpu
def test_vortex_gpu():
    _vortex_checks(_gpu())


@pytest.mark.gpu
def test_materials_gpu():
    _materials_checks(_gpu())
