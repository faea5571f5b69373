"""The workloads: seeded synthetic cases with the shapes of the reference's
benchmark configurations, and the crossing-jets case of its validation suite.

No dataset is involved: every field is generated here from a seed.
"""
from __future__ import annotations

import math

import numpy as np

from .case import Case, Family, Numerics, box_bc, box_nodes, empty_state

PI = 3.14159265358979323846


def particle_mass(radius, rho_m):
    return 4.0 / 3.0 * PI * radius ** 3 * rho_m


def _gas_layout(case: Case, b: int, rho, u, v, w, T, R=287.05, gam=1.4, k=0.026, mu=1.8e-5):
    ni, nj, nk = case.dims[b]
    shp = (nk, nj, ni)
    prim5 = np.stack([np.broadcast_to(rho, shp), np.broadcast_to(u, shp), np.broadcast_to(v, shp),
                      np.broadcast_to(w, shp), np.broadcast_to(T, shp)], axis=-1).astype(np.float64)
    full = lambda x: np.ascontiguousarray(np.broadcast_to(np.float64(x), shp))
    return {"prim5": np.ascontiguousarray(prim5), "R": full(R), "gam": full(gam), "k": full(k), "mu": full(mu)}


def fourier_velocity(rng, shape, spacing, lo, nmodes=32, kmin=1, kmax=8, rms=10.0, ndim=3, length=None):
    """A divergence-free sum of nmodes seeded Fourier modes at the cell centres, |k| in
    [kmin, kmax] (units of 2 pi / length), scaled to the given RMS speed. Returns (u, v, w)
    with shape (nk, nj, ni)."""
    nk, nj, ni = shape
    L = length
    xc = lo[0] + (np.arange(ni) + 0.5) * spacing[0]
    yc = lo[1] + (np.arange(nj) + 0.5) * spacing[1]
    zc = lo[2] + (np.arange(nk) + 0.5) * spacing[2]
    ks, amps, phases = [], [], []
    while len(ks) < nmodes:
        kv = rng.integers(-kmax, kmax + 1, size=3)
        if ndim == 2:
            kv[2] = 0
        kn = float(np.linalg.norm(kv))
        if kn < kmin or kn > kmax:
            continue
        a = rng.normal(size=3)
        if ndim == 2:
            a[2] = 0.0
        a = a - kv * (a @ kv) / (kn * kn)          # A . k = 0: divergence-free
        ks.append(kv); amps.append(a / max(np.linalg.norm(a), 1e-30) / kn); phases.append(rng.uniform(0, 2 * PI))
    u = np.zeros(shape); v = np.zeros(shape); w = np.zeros(shape)
    for kv, a, ph in zip(ks, amps, phases):
        arg = (2 * PI / L) * (kv[0] * xc[None, None, :] + kv[1] * yc[None, :, None] + kv[2] * zc[:, None, None]) + ph
        cs = np.cos(arg)
        u += a[0] * cs; v += a[1] * cs; w += a[2] * cs
    s = rms / math.sqrt(float(np.mean(u * u + v * v + w * w)))
    return u * s, v * s, w * s


def gaussian_blobs(rng, shape, spacing, lo, nblobs, width, length):
    nk, nj, ni = shape
    xc = lo[0] + (np.arange(ni) + 0.5) * spacing[0]
    yc = lo[1] + (np.arange(nj) + 0.5) * spacing[1]
    zc = lo[2] + (np.arange(nk) + 0.5) * spacing[2]
    out = np.zeros(shape)
    which = np.full(shape, -1, dtype=np.int64)
    best = np.zeros(shape)
    for m in range(nblobs):
        c = lo + rng.uniform(0.15, 0.85, size=3) * length
        g = (np.exp(-((xc[None, None, :] - c[0]) ** 2) / (2 * width ** 2))
             * np.exp(-((yc[None, :, None] - c[1]) ** 2) / (2 * width ** 2))
             * np.exp(-((zc[:, None, None] - c[2]) ** 2) / (2 * width ** 2)))
        out += g
        which = np.where(g > best, m, which)
        best = np.maximum(best, g)
    return np.minimum(out, 1.0), which


# ------------------------------------------------------------ config 1
def riemann_1d(n=2000, steps=1000):
    """Plain FP64 1-D IG Riemann problem: 2000 cells on [0,1], discontinuity at 0.5,
    left rho 1 u +1 theta 0.1, right rho 0.5 u -1 theta 0.05, 10 um particles of
    material density 1000, exchange off, transmissive ends. MUSCL minmod, HLLE, SSP-RK3,
    CFL 0.5. dt-max is set above the CFL step (1.0) so that the CFL condition sets dt."""
    dx = 1.0 / n
    nodes = box_nodes(n, 1, 1, size=(1.0, dx, dx))
    fam = Family("IG", riemann="HLLE", rho_al=1000.0, cs_al=1000.0)
    num = Numerics(scheme="RK3", cfl=0.5, dt_max=1.0, limiter="minmod", itermax=steps)
    rows = box_bc(1, (n, 1, 1), {1: 400, 2: 400, 3: 0, 4: 0, 5: 0, 6: 0})
    case = Case("riemann_1d", [nodes], [fam], num, rows)
    st = empty_state((n, 1, 1), 7)
    xc = (np.arange(n) + 0.5) * dx
    left = xc < 0.5
    rho = np.where(left, 1.0, 0.5)
    u = np.where(left, 1.0, -1.0)
    theta = np.where(left, 0.1, 0.05)
    mp = particle_mass(10e-6, 1000.0)
    I = st[2:3, 2:3, 2:-2]
    I[..., 0] = rho; I[..., 1] = u; I[..., 2] = 0.0; I[..., 3] = 0.0
    I[..., 4] = rho * theta; I[..., 5] = 300.0; I[..., 6] = rho / mp
    case.state = [[st]]
    return case


def ag_tube(ic, x0=-0.5, lx=1.0, ny=1, ly=1e-3, h=1e-3, side_code=0, scheme="RK2", limiter="mc", cfl=0.5,
            dt_max=1e-4, t_end=0.125, riemann="Rusanov", rho_al=2700.0, cs=1598.0):
    """A 1-D Riemann problem of the anisotropic Gaussian closure, the setting of the reference's Berthon
    cases (test/Berthon/*: 500 cells of [-0.5, 0.5], 1e-3 wide and thick, extrapolation at the ends,
    MUSCL with the MC limiter, RK2, CFL 0.5, material 2700 kg/m3, cp 1598) and of its anisotropic Sod
    tube (test/Riemann/AG). ic: the 12 AG primitives (rho, u, v, w, P11, P12, P13, P22, P23, P33, T, n)
    per cell along x, shape (12, nx), repeated over the ny rows; side_code: the boundary code of the
    j faces (0 none, 300 wall); the k faces are 0. No gas; the run ends at time >= t_end."""
    ic = np.asarray(ic, dtype=np.float64)
    nx = ic.shape[1]
    nodes = box_nodes(nx, ny, 1, lo=(x0, 0.0, -0.5 * h), size=(lx, ly, h))
    fam = Family("AG", riemann=riemann, rho_al=rho_al, cs_al=cs)
    num = Numerics(scheme=scheme, cfl=cfl, dt_max=dt_max, limiter=limiter, time_threshold=t_end)
    rows = box_bc(1, (nx, ny, 1), {1: 400, 2: 400, 3: side_code, 4: side_code, 5: 0, 6: 0})
    case = Case("ag_tube", [nodes], [fam], num, rows)
    st = empty_state((nx, ny, 1), 12)
    st[2, 2:-2, 2:-2, :] = ic.T[None, :, :]
    case.state = [[st]]
    return case


def _cell_centres(nodes):
    """Cell centres as the mean of the 8 corner nodes, arrays (ni, nj, nk) per coordinate."""
    c = sum(nodes[a:a + nodes.shape[0] - 1, b:b + nodes.shape[1] - 1, d:d + nodes.shape[2] - 1]
            for a in (0, 1) for b in (0, 1) for d in (0, 1)) / 8.0
    return c[..., 0], c[..., 1], c[..., 2]


def _single_block(name, nodes, fam, num, codes, prims, payload=None):
    """One block with the given boundary codes per face and the interior primitives prims (a list of
    nc arrays or scalars over the (ni, nj, nk) cells)."""
    dims = tuple(s - 1 for s in nodes.shape[:3])
    case = Case(name, [nodes], [fam], num, box_bc(1, dims, codes, payload))
    st = empty_state(dims, fam.nc)
    for q, a in enumerate(prims):
        st[2:-2, 2:-2, 2:-2, q] = np.broadcast_to(a, dims).transpose(2, 1, 0)
    case.state = [[st]]
    return case


def noexchange_slab(precision=0):
    """The reference's no-exchange invariant case (test/NoExchange/MK): 10 x 4 cells of a 0.1 x 0.04 m
    slab 1 mm thick, an MK cloud at rest at 300 K (1e-3 kg/m3 of 1 um drops of material density 2000,
    cp 1000) in a gas at 10 m/s and 400 K (1.0 kg/m3, R 287, gamma 1.4, k 0.025, mu 2e-5), coupled with
    NoDrag, NoHeat and no emissivity; extrapolation on the i and j faces, RK3, CFL 0.8, MUSCL van Leer,
    20 steps. Nothing couples the phases, so the state stays at its initial value exactly."""
    nodes = box_nodes(10, 4, 1, lo=(0.0, 0.0, -0.5e-3), size=(0.1, 0.04, 1e-3))
    fam = Family("MK", rho_al=2000.0, cs_al=1000.0)
    num = Numerics(scheme="RK3", cfl=0.8, limiter="vanleer", coupled=True, drag="NoDrag", heat="NoHeat",
                   itermax=20, precision=precision)
    n = 1e-3 / particle_mass(1e-6, 2000.0)
    case = _single_block("noexchange_slab", nodes, fam, num, {1: 400, 2: 400, 3: 400, 4: 400, 5: 0, 6: 0},
                         [1e-3, 0.0, 0.0, 0.0, 300.0, n])
    case.gas = [_gas_layout(case, 0, 1.0, 10.0, 0.0, 0.0, 400.0, R=287.0, gam=1.4, k=0.025, mu=2e-5)]
    return case


def reflect_blob(precision=0):
    """The reference's symmetry-plane case of the AG closure (test/Reflect/AG): 200 x 100 cells of
    [0, 2] x [0, 1], 0.01 thick; the upper half of a sheared AG blob, rho = 0.01 + g with
    g = exp(-((x - 1)^2 + y^2) / (2 0.1^2)), moving at u = 1 along the code-200 plane y = 0 (face 3);
    P11 = P22 = P33 = rho, P12 = 0.3 g y / 0.1, T = 1, 1 um drops of material density 2000, cp 1; faces 1,
    2 and 4 extrapolation. RK3, CFL 0.8, MUSCL van Leer, dt-max 1e-2, to t = 0.1. The mirrored tensor
    exerts no shear on the plane, so the x-momentum is conserved."""
    nodes = box_nodes(200, 100, 1, lo=(0.0, 0.0, -0.005), size=(2.0, 1.0, 0.01))
    x, y, _ = _cell_centres(nodes)
    blob = np.exp(-((x - 1.0) ** 2 + y ** 2) / (2.0 * 0.1 ** 2))
    rho = 0.01 + blob
    fam = Family("AG", riemann="Rusanov", rho_al=2000.0, cs_al=1.0)
    num = Numerics(scheme="RK3", cfl=0.8, dt_max=1e-2, limiter="vanleer", time_threshold=0.1,
                   precision=precision)
    return _single_block("reflect_blob", nodes, fam, num, {1: 400, 2: 400, 3: 200, 4: 400, 5: 0, 6: 0},
                         [rho, 1.0, 0.0, 0.0, rho, 0.3 * blob * y / 0.1, 0.0, rho, 0.0, rho, 1.0,
                          rho / particle_mass(1e-6, 2000.0)])


def thermal_blob(closure="IG", precision=0):
    """The reference's thermal-energy invariant cases (test/Thermal/{IG,AG}): a pressurised blob
    rho = 0.01 + exp(-((x - 0.5)^2 + (y - 0.5)^2) / (2 0.05^2)) at rest, P = rho (isotropic for AG), T = 1,
    1 um drops of material density 2000 and cp 1, in a closed box of 100 x 100 cells of [0, 1]^2, 0.01
    thick (walls, code 300, on the four sides). RK3, CFL 0.5 (IG) or 0.8 (AG), MUSCL van Leer, dt-max
    1e-2, to t = 0.1. With the pressure work in the energy flux the temperature stays uniform."""
    nodes = box_nodes(100, 100, 1, lo=(0.0, 0.0, -0.005), size=(1.0, 1.0, 0.01))
    x, y, _ = _cell_centres(nodes)
    rho = 0.01 + np.exp(-((x - 0.5) ** 2 + (y - 0.5) ** 2) / (2.0 * 0.05 ** 2))
    n = rho / particle_mass(1e-6, 2000.0)
    fam = Family(closure, riemann="Rusanov", rho_al=2000.0, cs_al=1.0)
    num = Numerics(scheme="RK3", cfl=0.5 if closure == "IG" else 0.8, dt_max=1e-2, limiter="vanleer",
                   time_threshold=0.1, precision=precision)
    prims = ([rho, 0.0, 0.0, 0.0, rho, 1.0, n] if closure == "IG" else
             [rho, 0.0, 0.0, 0.0, rho, 0.0, 0.0, rho, 0.0, rho, 1.0, n])
    return _single_block("thermal_blob", nodes, fam, num, {1: 300, 2: 300, 3: 300, 4: 300, 5: 0, 6: 0}, prims)


def axis_wedge(closure="MK", precision=0):
    """The reference's axisymmetric-wedge cases (test/Axis/{MK,IG,AG}): a one-degree wedge about x,
    40 x 20 cells of x in [0, 0.1], r in [1e-8, 0.05] (the axis row at r = 1e-8, face 3, code 300), the
    wedge sides (faces 5, 6) code 200; drops of 10 um, material density 2000, cp 1000, T 300.
    MK: a cloud moving along x at 20 m/s with rho = 1 + 4 (r / 0.05)^2, fed through face 1 by a 402 inlet
    of the same profile along the face normal; face 2 extrapolation, face 4 a wall; RK3, MUSCL van Leer
    with the Jameson sensor, CFL 0.8, local steps, 200 iterations: the field is stationary.
    IG, AG: a uniform cloud at rest (rho 1, P = 1, isotropic for AG) closed by walls on faces 1-4; RK2,
    MUSCL van Leer, CFL 0.8, local steps, 500 iterations: the side faces carry the hoop pressure and
    the cloud stays at rest."""
    x = np.linspace(0.0, 0.1, 41)
    r = np.linspace(1e-8, 0.05, 21)
    th = np.radians([-0.5, 0.5])
    X, R, T = np.meshgrid(x, r, th, indexing="ij")
    nodes = np.stack([X, R * np.cos(T), R * np.sin(T)], axis=-1)
    _, yc, zc = _cell_centres(nodes)
    mk = closure == "MK"
    fam = Family(closure, rho_al=2000.0, cs_al=1000.0)
    num = Numerics(scheme="RK3" if mk else "RK2", cfl=0.8, limiter="vanleer", shock_detector=mk,
                   time_accurate=False, itermax=200 if mk else 500, precision=precision)
    mp = particle_mass(1e-5, 2000.0)
    if mk:
        rho = 1.0 + 4.0 * (np.sqrt(yc ** 2 + zc ** 2) / 0.05) ** 2
        prims = [rho, 20.0, 0.0, 0.0, 300.0, rho / mp]
        codes = {1: 402, 2: 400, 3: 300, 4: 300, 5: 200, 6: 200}
        payload = lambda f, i, j, k: (rho[0, j - 1, k - 1] * 20.0, 20.0, 0.0, 0.0, 300.0, 1e-5, 0.0, 1.0)
    else:
        prims = ([1.0, 0.0, 0.0, 0.0, 1.0, 300.0, 1.0 / mp] if closure == "IG" else
                 [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 1.0, 0.0, 1.0, 300.0, 1.0 / mp])
        codes = {1: 300, 2: 300, 3: 300, 4: 300, 5: 200, 6: 200}
        payload = None
    return _single_block("axis_wedge", nodes, fam, num, codes, prims, payload)


def mirror_layer(kind="slab", closure="IG", side_code=300):
    """The reference's mirror-modes cases (test/fast/mirror-modes): a cloud at rest (rho 1, P = 1, T 300,
    10 um drops of density 2000, cp 1000) whose components odd across the mirror faces start at 1e-8 of
    the signal speed: s = 1e-8 sin(2 pi x / L) cos(pi y / H_y), w = sqrt(3) s (AG: P13 = P23 = s; the tube
    also v = sqrt(3) s, AG P12 = s), every face code 300 (a wall); RK2, CFL 0.8, dt-max 1e3, local steps,
    MUSCL van Leer, 200 steps. slab: 16 x 8 cells of 2.5 mm, 1e-5 m thick; tube: 32 cells along 0.04 m,
    1e-5 m across; wedge: the slab's x and 8 radial cells from r = 1e-8 to 0.02 turned by one degree, its
    k faces carrying side_code."""
    h, n_x, n_y, length = 1e-5, 16, 8, 0.04
    if kind == "tube":
        nodes = box_nodes(2 * n_x, 1, 1, lo=(0.0, -0.5 * h, -0.5 * h), size=(length, h, h))
    elif kind == "slab":
        nodes = box_nodes(n_x, n_y, 1, lo=(0.0, 0.0, -0.5 * h), size=(length, 0.5 * length, h))
    else:
        X, R, T = np.meshgrid(np.linspace(0.0, length, n_x + 1), np.linspace(1e-8, 0.5 * length, n_y + 1),
                              np.radians([-0.5, 0.5]), indexing="ij")
        nodes = np.stack([X, R * np.cos(T), R * np.sin(T)], axis=-1)
    x, y, _ = _cell_centres(nodes)
    y0, y1 = float(nodes[..., 1].min()), float(nodes[:, -1, 0, 1].max())
    s = 1e-8 * np.sin(2.0 * math.pi * x / length) * np.cos(math.pi * (y - y0) / (y1 - y0))
    odd_v = kind == "tube"
    c = math.sqrt(3.0)
    w = c * s if kind != "wedge" else 0.0 * s
    v = c * s if odd_v else 0.0 * s
    n = 1.0 / particle_mass(1e-5, 2000.0)
    fam = Family(closure, rho_al=2000.0, cs_al=1000.0)
    num = Numerics(scheme="RK2", cfl=0.8, dt_max=1e3, limiter="vanleer", time_accurate=False, itermax=200)
    codes = {f: 300 for f in range(1, 7)}
    if kind == "wedge":
        codes[5] = codes[6] = side_code
    if closure == "IG":
        prims = [1.0, 0.0, v, w, 1.0, 300.0, n]
    else:
        odd = kind != "wedge"
        prims = [1.0, 0.0, v, w, 1.0, s if odd_v else 0.0 * s, s if odd else 0.0 * s, 1.0,
                 s if odd else 0.0 * s, 1.0, 300.0, n]
    return _single_block("mirror_layer", nodes, fam, num, codes, prims)


def inlet_duct(kind="normal"):
    """The reference's inlet-direction case (test/fast/inlet-direction): a 1-D duct of 16 cells along
    0.16 m, an MK cloud at rest (1e-3 kg/m3 of 10 um drops of density 1000, 300 K), extrapolation on the
    i and j faces, the inlet on face 2 (x = 0.16, whose normal points out of the domain); RK2, CFL 0.5,
    NoDrag, NoHeat, 200 steps. normal: a 402 inlet of 1 kg/(s m2) at 10 m/s along the face normal, 300 K,
    10 um, no gas. angles: a 401 inlet (mass ratio 1, kV = kT = 1) with explicit angles alpha = 180 deg,
    beta = 0, in a gas (1.2 kg/m3, 300 K) moving along -x at 10 m/s."""
    nx, lx = 16, 0.16
    nodes = box_nodes(nx, 1, 1, size=(lx, lx / nx, lx / nx))
    fam = Family("MK", rho_al=1000.0, cs_al=900.0)
    num = Numerics(scheme="RK2", cfl=0.5, limiter="vanleer", coupled=kind == "angles", drag="NoDrag",
                   heat="NoHeat", itermax=200)
    mass = particle_mass(1e-5, 1000.0)
    if kind == "normal":
        code, pay = 402, (1.0, 10.0, 0.0, 0.0, 300.0, 1e-5, 0.0, 1.0)
    else:
        code, pay = 401, (1.0, 1.0, math.pi, 0.0, 1.0, 1e-5, 0.0, 0.0)
    case = _single_block("inlet_duct", nodes, fam, num, {1: 400, 2: code, 3: 400, 4: 400, 5: 0, 6: 0},
                         [1e-3, 0.0, 0.0, 0.0, 300.0, 1e-3 / mass], lambda f, i, j, k: pay)
    if kind == "angles":
        case.gas = [_gas_layout(case, 0, 1.2, -10.0, 0.0, 0.0, 300.0)]
    return case


def population_duct(copies=3, families=3, scaled=True):
    """The reference's populations case (test/fast/populations): a duct of 16 x 4 cells over 0.16 x 0.04 m,
    MK families of 10 um drops (density 1000) at rest at 300 K, loaded 1e-3 kg/m3 (times 2^(p-1) for
    family p when scaled); a 402 inlet on face 1 (10 m/s along the normal, 300 K, 10 um) whose mass flux is
    2 kg/(s m2) times 2^c in copy c of the boundary table; extrapolation on faces 2-4; RK2, CFL 0.8,
    30 steps, no gas."""
    mass = particle_mass(1e-5, 1000.0)
    nodes = box_nodes(16, 4, 1, size=(0.16, 0.04, 0.01))
    fam = Family("MK", rho_al=1000.0, cs_al=900.0)
    num = Numerics(scheme="RK2", cfl=0.8, limiter="vanleer", itermax=30)
    codes = {1: 402, 2: 400, 3: 400, 4: 400, 5: 0, 6: 0}
    tables = [box_bc(1, (16, 4, 1), codes, lambda f, i, j, k, c=c: (2.0 * 2.0 ** c, 10.0, 0.0, 0.0, 300.0, 1e-5,
                                                                     0.0, 1.0))
              for c in range(copies)]
    case = _single_block("population_duct", nodes, fam, num, codes, [1e-3, 0.0, 0.0, 0.0, 300.0, 1e-3 / mass])
    case.bc_rows = tables[0]
    case.bc_copies = tables
    st = case.state[0][0]
    case.families = [Family("MK", rho_al=1000.0, cs_al=900.0) for _ in range(families)]
    per_fam = []
    for p in range(families):
        q = st.copy()
        if scaled:
            q[..., 0] *= 2.0 ** p
            q[..., 5] *= 2.0 ** p
        per_fam.append(q)
    case.state = [per_fam]
    return case


def stream_tube(kind="scaling", scale=1.0):
    """The reference's res-threshold cases (test/fast/res-threshold), steady (local steps), res-threshold
    1e-5, MK drops of 10 um and density 1000 at 300 K, extrapolation on every face but the inlet.
    scaling: 32 cells along 0.32 m, rho = scale (1 + 0.5 sin(2 pi x / 0.32)) moving at 10 m/s, fed through
    face 1 by a 402 inlet of scale x 10 kg/(s m2) at 10 m/s along the normal; RK2, CFL 0.8, NoDrag, NoHeat.
    at_rest: the same density at rest in a uniform gas at 10 m/s (1.2 kg/m3, 300 K), Stokes drag and
    heat, one-stage Euler steps, no inlet. frozen: 16 cells along 0.16 m of a uniform cloud (1 kg/m3)
    moving at 10 m/s out through face 2; RK2, 40 iterations."""
    mass = particle_mass(1e-5, 1000.0)
    nx, lx = (16, 0.16) if kind == "frozen" else (32, 0.32)
    nodes = box_nodes(nx, 1, 1, size=(lx, lx / nx, lx / nx))
    fam = Family("MK", rho_al=1000.0, cs_al=900.0)
    num = Numerics(scheme="euler" if kind == "at_rest" else "RK2", cfl=0.8, limiter="vanleer",
                   time_accurate=False, coupled=kind == "at_rest",
                   drag="Stokes" if kind == "at_rest" else "NoDrag", heat="Stokes" if kind == "at_rest" else "NoHeat",
                   itermax=40 if kind == "frozen" else 20000, res_threshold=1e-5)
    x = (np.arange(nx) + 0.5) * (lx / nx)
    rho = np.ones(nx) if kind == "frozen" else scale * (1.0 + 0.5 * np.sin(2.0 * math.pi * x / lx))
    u = 0.0 if kind == "at_rest" else 10.0
    codes = {1: 402 if kind == "scaling" else 400, 2: 400, 3: 400, 4: 400, 5: 0, 6: 0}
    pay = (scale * 10.0, 10.0, 0.0, 0.0, 300.0, 1e-5, 0.0, 1.0)
    prims = [rho[:, None, None], u, 0.0, 0.0, 300.0, (rho / mass)[:, None, None]]
    case = _single_block("stream_tube", nodes, fam, num, codes, prims, lambda f, i, j, k: pay)
    if kind == "at_rest":
        case.gas = [_gas_layout(case, 0, 1.2, 10.0, 0.0, 0.0, 300.0)]
    return case


def empty_tube(n_occupied=2, time_accurate=False, narrow_last=False, steps=1):
    """The setting of the reference's unit test of the steps of empty cells a source fills
    (test/unit/test_empty_dt.f90): one block of 4 x 1 x 1 cells of 1 mm (the last 0.1 mm wide when
    narrow_last), an MK family, CFL 0.4, dt-max 1e-4 s; the first n_occupied cells at density 1 and
    100 m/s (300 K, 1e9 particles), the others at ICE's empty state (1e-25 in every slot); transmissive
    ends. The coupler's imports are set separately (ice_gpu_set_imports)."""
    dx = 1e-3
    x = np.array([0.0, 1.0, 2.0, 3.0, 3.1 if narrow_last else 4.0]) * dx
    X, Y, Z = np.meshgrid(x, np.array([0.0, dx]), np.array([0.0, dx]), indexing="ij")
    nodes = np.stack([X, Y, Z], axis=-1)
    fam = Family("MK", rho_al=1000.0, cs_al=1000.0)
    num = Numerics(scheme="euler", time_accurate=time_accurate, cfl=0.4, dt_max=1e-4, limiter="minmod",
                   itermax=steps)
    rows = box_bc(1, (4, 1, 1), {1: 400, 2: 400, 3: 0, 4: 0, 5: 0, 6: 0})
    case = Case("empty_tube", [nodes], [fam], num, rows)
    st = empty_state((4, 1, 1), 6)
    I = st[2:3, 2:3, 2:-2]
    I[...] = 1e-25
    I[0, 0, :n_occupied] = [1.0, 100.0, 0.0, 0.0, 300.0, 1e9]
    case.state = [[st]]
    return case


def relaxation_tube(nx=8, ny=1, lx=1.0, ly=None, scheme="RK2", cfl=0.8, dt_max=1e-4, vg=0.0, steps=1,
                    drag="Stokes", heat="Stokes", precision=0, up0=0.0, tp0=300.0, ug=10.0, lz=None,
                    dp=1e-4, rho_al=1000.0, cs=900.0, rho_g=1.2, mu=1.8e-5, kg=0.026, tau_factor=1.0):
    """The setting of the reference's drag-relaxation verification case (test/verification/
    A-drag-relaxation): a uniform MK cloud (1e-4 m drops of material density 1000, cp 900, volume
    fraction 1e-3) at rest in a uniform gas stream (1.2 kg/m3, ug along x and vg along y, 300 K,
    R 287.05, gamma 1.4, mu 1.8e-5, k 0.026), one-way coupled with the given drag and heat laws,
    nx x ny cells of a slab lx long (ly wide: square cells by default), extrapolation on every face.
    With no gradient anywhere the particle velocity relaxes as u_g + (u_p0 - u_g) exp(-t/tau) with
    tau = rho_al dp^2 / (18 mu) under Stokes drag, and density, number density and temperature stay.
    With up0 = 10 (no slip) and tp0 = 400 it is the thermal-relaxation case (test/verification/
    B-thermal-relaxation): T_g + (T_p0 - T_g) exp(-t/tau_T), tau_T = rho_al cs dp^2 / (12 k), Nu = 2.
    dp, rho_al, cs (the drops) and rho_g, mu, kg (the gas) change the defaults above; tau_factor is the
    step's bound by the relaxation time (the reference's tau-factor)."""
    ly = lx / nx * ny if ly is None else ly
    dz = lx / nx if lz is None else lz
    nodes = box_nodes(nx, ny, 1, size=(lx, ly, dz))
    fam = Family("MK", rho_al=rho_al, cs_al=cs)
    num = Numerics(scheme=scheme, cfl=cfl, dt_max=dt_max, limiter="vanleer", coupled=True, drag=drag,
                   heat=heat, itermax=steps, precision=precision, tau_factor=tau_factor)
    rows = box_bc(1, (nx, ny, 1), {f: 400 for f in range(1, 7)} if ny > 1 else
                  {1: 400, 2: 400, 3: 0, 4: 0, 5: 0, 6: 0})
    if ny > 1:
        rows = [(b, i, j, k, f, 0 if f >= 5 else code, pay) for (b, i, j, k, f, code, pay) in rows]
    case = Case("relaxation_tube", [nodes], [fam], num, rows)
    rho_p = 1e-3 * rho_al
    n = rho_p / particle_mass(0.5 * dp, rho_al)
    st = empty_state((nx, ny, 1), 6)
    st[2:-2, 2:-2, 2:-2, :] = [rho_p, up0, vg, 0.0, tp0, n]
    case.state = [[st]]
    case.gas = [_gas_layout(case, 0, rho_g, ug, vg, 0.0, 300.0, k=kg, mu=mu)]
    return case


def periodic_sine(nx=50, limiter="vanleer", steps=2500, scheme="RK2", precision=0):
    """The setting of the reference's periodic sine-advection verification case (test/verification/
    C-advection-sine): a pressureless MK cloud (1e-4 m drops of material density 1000) moving at 1 m/s
    through nx cells of [0, 1] joined end to end (periodic connections, 201), no gas, density
    10 + 5 sin(2 pi x) with the number density of 1e-4 m drops; CFL 0.8 under the default dt-max 1e-4 s,
    so dt is 1e-4 on every grid. Free transport shifts the profile by the distance travelled.
    limiter: "vanleer" (MUSCL) or "IORD" (first-order reconstruction)."""
    dx = 1.0 / nx
    nodes = box_nodes(nx, 1, 1, size=(1.0, dx, dx))
    fam = Family("MK", rho_al=1000.0, cs_al=900.0)
    num = Numerics(scheme=scheme, cfl=0.8, limiter=limiter, coupled=False, itermax=steps, precision=precision)
    rows = []
    for f, i0, src, fs in ((1, 1, nx, 2), (2, nx, 1, 1)):
        rows.append((1, i0, 1, 1, f, 201, (1, src, 1, 1, fs)))
    for f in (3, 4):
        for i in range(1, nx + 1):
            rows.append((1, i, 1, 1, f, 400, ()))
    for f in (5, 6):
        for i in range(1, nx + 1):
            rows.append((1, i, 1, 1, f, 0, ()))
    case = Case("periodic_sine", [nodes], [fam], num, rows)
    x = (np.arange(nx) + 0.5) * dx
    k = 2.0 * PI
    # the cell averages of 10 + 5 sin(k x)
    rho = 10.0 + 5.0 * (np.cos(k * (x - 0.5 * dx)) - np.cos(k * (x + 0.5 * dx))) / (k * dx)
    st = empty_state((nx, 1, 1), 6)
    I = st[2:3, 2:3, 2:-2]
    I[0, 0, :, 0] = rho; I[0, 0, :, 1] = 1.0; I[0, 0, :, 2] = 0.0; I[0, 0, :, 3] = 0.0
    I[0, 0, :, 4] = 300.0; I[0, 0, :, 5] = rho / particle_mass(0.5e-4, 1000.0)
    case.state = [[st]]
    return case


def evaporating_tube(model="CEM", interface="VLE", steps=2000, cs=1e12, dt_max=2e-5, precision=0, blowing=False,
                     tp0=300.0):
    """The setting of the reference's droplet-evaporation verification case, part 1 (test/verification/
    F-evaporation): water droplets of 1e-4 m at volume fraction 1e-3, at rest at 300 K in air at rest at
    800 K and one atmosphere, 8 cells of a slab, the given evaporation model and interface (VLE or LK),
    drag and heat Stokes, no blowing correction, RK2, CFL 0.8, dt-max 2e-5 s. The default specific heat
    (1e12) freezes the droplet temperature, so d^2 falls linearly in time (the d-squared law); cs 4180
    releases it; blowing switches the Miller-Harstad-Bellan correction on; tp0 the droplet temperature."""
    nx = 8
    nodes = box_nodes(nx, 1, 1, size=(1.0, 1.0 / nx, 1.0 / nx))
    fam = Family("MK", rho_al=1000.0, cs_al=cs, lv_al=2.26e6, emiss=0.0, evap=model, intf=interface,
                 Mv=18.015, cpv=0.0, Le=1.0, Yinf=0.0, Tboil=373.15, alphaE=1.0)
    num = Numerics(scheme="RK2", cfl=0.8, dt_max=dt_max, limiter="vanleer", coupled=True, drag="Stokes",
                   heat="Stokes", blowing=blowing, itermax=steps, precision=precision)
    rows = box_bc(1, (nx, 1, 1), {1: 400, 2: 400, 3: 0, 4: 0, 5: 0, 6: 0})
    case = Case("evaporating_tube", [nodes], [fam], num, rows)
    n = 1.0 / particle_mass(0.5e-4, 1000.0)
    st = empty_state((nx, 1, 1), 6)
    st[2:-2, 2:-2, 2:-2, :] = [1.0, 0.0, 0.0, 0.0, tp0, n]
    case.state = [[st]]
    case.gas = [_gas_layout(case, 0, 101325.0 / (287.05 * 800.0), 0.0, 0.0, 0.0, 800.0)]
    return case


def with_families(case, families):
    """The case with the given families in place of its one, each starting from the first family's
    initial state (the reference's several-materials cases, test/verification/L-materials: one family
    per material line, each reading its own material)."""
    st = case.state[0][0]
    case.families = list(families)
    case.state = [[st.copy() for _ in case.families]]
    return case


def cloud_profile(shape, x):
    """The bulk-density profile of periodic_cloud at x in [0, 1): 10 (s(x) + 1e-6), s a Gaussian of
    width 0.06 about 0.25 summed over its periodic images ("gauss"), or a top hat of half width 0.1
    about 0.25 ("tophat")."""
    x = np.asarray(x, dtype=np.float64)
    if shape == "gauss":
        s = sum(np.exp(-(x - 0.25 - m) ** 2 / (2.0 * 0.06 ** 2)) for m in (-1, 0, 1))
    else:
        d = (x - 0.25 + 0.5) % 1.0 - 0.5
        s = np.where(np.abs(d) <= 0.1, 1.0, 0.0)
    return 10.0 * (s + 1e-6)


def periodic_cloud(nx=100, shape="gauss", dt_max=1e-5, steps=1, precision=0):
    """The setting of the reference's cloud-translation verification case (test/verification/
    G-cloud-translation): a cloud of 1e-4 m MK drops (material density 1000, cp 900) at rest, its bulk
    density cloud_profile(shape) sampled at the cell centres of a periodic slab of nx cells (201
    connections), number density proportional to it (one diameter everywhere), released into a frozen
    uniform gas at 10 m/s (1.2 kg/m3, 300 K, mu 1.8e-5) with Stokes drag and heat; CFL 0.4 under dt-max.
    The drops relax as u_p = 10 (1 - exp(-t/tau)) and the cloud translates rigidly by
    10 t - 10 tau (1 - exp(-t/tau))."""
    case = periodic_sine(nx, "vanleer", steps, "RK2", precision)
    case.name = "periodic_cloud"
    case.numerics.cfl = 0.4
    case.numerics.dt_max = dt_max
    case.numerics.coupled = True
    case.numerics.drag = "Stokes"
    case.numerics.heat = "Stokes"
    dx = 1.0 / nx
    rho = cloud_profile(shape, (np.arange(nx) + 0.5) * dx)
    st = empty_state((nx, 1, 1), 6)
    I = st[2:3, 2:3, 2:-2]
    I[0, 0, :, 0] = rho; I[0, 0, :, 1] = 0.0; I[0, 0, :, 2] = 0.0; I[0, 0, :, 3] = 0.0
    I[0, 0, :, 4] = 300.0; I[0, 0, :, 5] = rho / particle_mass(0.5e-4, 1000.0)
    case.state = [[st]]
    case.gas = [_gas_layout(case, 0, 1.2, 10.0, 0.0, 0.0, 300.0)]
    return case


def strain_tube(nx=100, dp=1e-4, steps=1, precision=0):
    """The setting of the reference's linear-strain verification case (test/verification/
    H-linear-strain): a frozen gas (1.2 kg/m3, 300 K, mu 1.8e-5) in the uniform strain u_g = 2 + 6 x on
    nx cells of [0, 1], extrapolation on every face; a Gaussian cloud 10 (exp(-(x - 0.2)^2 / (2 0.035^2))
    + 1e-6) sampled at the cell centres, seeded at the local gas velocity, with the number density of
    drops of diameter dp (material density 1000, cp 900); Stokes drag and heat, CFL 0.4, dt-max 2e-5.
    With xi = x + 1/3 every drop is displaced by one factor C(t), so the solution is the affine map
    rho_p(x, t) = rho_p0(xi / C - 1/3) / C, u_p = (C'/C) xi."""
    case = relaxation_tube(nx=nx, cfl=0.4, dt_max=2e-5, steps=steps, precision=precision, dp=dp)
    case.name = "strain_tube"
    x = (np.arange(nx) + 0.5) / nx
    rho = 10.0 * (np.exp(-(x - 0.2) ** 2 / (2.0 * 0.035 ** 2)) + 1e-6)
    ug = 2.0 + 6.0 * x
    st = empty_state((nx, 1, 1), 6)
    I = st[2:3, 2:3, 2:-2]
    I[0, 0, :, 0] = rho; I[0, 0, :, 1] = ug; I[0, 0, :, 2] = 0.0; I[0, 0, :, 3] = 0.0
    I[0, 0, :, 4] = 300.0; I[0, 0, :, 5] = rho / particle_mass(0.5 * dp, 1000.0)
    case.state = [[st]]
    case.gas = [_gas_layout(case, 0, 1.2, ug, 0.0, 0.0, 300.0)]
    return case


def vortex_box(n=96, tau=0.1, steps=1, precision=0):
    """The setting of the reference's vortex-cloud verification case (test/verification/I-vortex-cloud):
    a frozen gas (1.2 kg/m3, 300 K, mu 1.8e-5) in solid-body rotation u_g = -y, v_g = x on n x n cells of
    [-2, 2]^2 (cells 4/n thick), extrapolation on every side; a Gaussian cloud 10 (exp(-((x - 0.6)^2 +
    y^2) / (2 0.12^2)) + 1e-8) sampled at the cell centres, seeded at the local gas velocity, with the
    number density of drops whose Stokes time is tau (material density 1000, cp 900); Stokes drag and
    heat, CFL 0.4, dt-max 1e-3. In z = x + i y every drop is displaced by one complex factor C(t), so
    rho_p(z, t) = rho_p0(z / C) / |C|^2 and u_p + i v_p = (C'/C) z."""
    dp = math.sqrt(18.0 * 1.8e-5 * tau / 1000.0)
    case = relaxation_tube(nx=n, ny=n, lx=4.0, ly=4.0, lz=4.0 / n, cfl=0.4, dt_max=1e-3, steps=steps,
                           precision=precision, dp=dp)
    case.name = "vortex_box"
    case.nodes = [box_nodes(n, n, 1, lo=(-2.0, -2.0, 0.0), size=(4.0, 4.0, 4.0 / n))]
    c = -2.0 + (np.arange(n) + 0.5) * (4.0 / n)
    Y, X = np.meshgrid(c, c, indexing="ij")
    rho = 10.0 * (np.exp(-((X - 0.6) ** 2 + Y ** 2) / (2.0 * 0.12 ** 2)) + 1e-8)
    st = empty_state((n, n, 1), 6)
    I = st[2, 2:-2, 2:-2]
    I[:, :, 0] = rho; I[:, :, 1] = -Y; I[:, :, 2] = X; I[:, :, 3] = 0.0
    I[:, :, 4] = 300.0; I[:, :, 5] = rho / particle_mass(0.5 * dp, 1000.0)
    case.state = [[st]]
    case.gas = [_gas_layout(case, 0, 1.2, -Y, X, 0.0, 300.0)]
    return case


# --------------------------------------------------- crossing jets (validation)
def crossing_jets(closure="IG", n=100, steps=5000, upper=None):
    """The crossing-jets validation case of the reference's suite (its Doisneau cases):
    100 x 100 cells of 0.01 on [0,1] x [-0.5,0.5], slab 1e-3 thick; face 1 symmetry except
    two inlets of 10 cells each (402: mass flux 0.7071, 10 m/s at +/-45 deg, 300 K, 1 um;
    j = 21..30 and 71..80, the MK case's upper inlet at 72..81 as its table has it),
    faces 2-4 extrapolation; every cell starts at 1e-20; steady (each cell its own dt),
    RK2, CFL 0.8, MUSCL van Leer, no exchange; constant material density 2000, cp 1500."""
    # the node coordinates are the decimal values of the case's mesh file, each parsed to
    # its nearest double, so that the mesh is symmetric about y = 0 to the bit
    dec = lambda a: np.array([float(f"{v:.8f}") for v in a])
    x = dec(np.arange(n + 1) / n)
    y = dec(np.arange(n + 1) / n - 0.5)
    z = np.array([-0.0005, 0.0005])
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    nodes = np.stack([X, Y, Z], axis=-1)
    fam = Family(closure, rho_al=2000.0, cs_al=1500.0)
    num = Numerics(scheme="RK2", time_accurate=False, cfl=0.8, limiter="vanleer", itermax=steps)

    def payload(f, i, j, k):
        alpha = 7.85400e-01 if j <= n // 2 else -7.85400e-01
        return (7.07100e-01, 1.0e1, alpha, 0.0, 3.0e2, 1.0e-6, 0.0, 0.0)
    codes = {1: 300, 2: 400, 3: 400, 4: 400, 5: 0, 6: 0}
    if upper is None:
        upper = (72, 81) if closure == "MK" else (71, 80)
    rows = []
    for row in box_bc(1, (n, n, 1), codes, face_major=True):
        b, i, j, k, f, code, pay = row
        if f == 1 and (21 <= j <= 30 or upper[0] <= j <= upper[1]):
            rows.append((b, i, j, k, f, 402, payload(f, i, j, k)))
        else:
            rows.append(row)
    case = Case(f"crossing_jets_{closure}", [nodes], [fam], num, rows)
    st = empty_state((n, n, 1), fam.nc)
    st[2:-2, 2:-2, 2:-2, :] = 1e-20
    case.state = [[st]]
    return case


def doisneau_chimera(data, closure="IG", steps=5000):
    """The overlapping-grid variant of the crossing-jets case in the reference's suite (its
    Doisneau IG-chimera case): block 1, 50 x 100 cells on [0,0.5] x [-0.5,0.5], and block 2,
    45 x 73 cells on [0.4,1] x [-0.5,0.5], overlap by 0.1 and meet at chimera faces (102) whose
    ghost cells blend donor cells of the other block; inlets, symmetry faces, numerics and
    material of the crossing-jets case. `data` holds the case's tables (a mapping of arrays as
    tests/golden/make_golden.py writes them from the case's mesh and boundary files): x<b>, y<b>,
    z<b> the node coordinates of block b, bc the rows b i j k f code, inlet the six inlet reals of
    each row, nchi the donors per ghost layer of each row, donor (b i j k) and weight."""
    nodes = []
    for b in (1, 2):
        X, Y, Z = np.meshgrid(data[f"x{b}"], data[f"y{b}"], data[f"z{b}"], indexing="ij")
        nodes.append(np.stack([X, Y, Z], axis=-1))
    fam = Family(closure, rho_al=2000.0, cs_al=1500.0)
    num = Numerics(scheme="RK2", time_accurate=False, cfl=0.8, limiter="vanleer", itermax=steps)
    rows, chim, off = [], {}, 0
    donor, weight = data["donor"], data["weight"]
    for n, (r, pay, nc) in enumerate(zip(data["bc"], data["inlet"], data["nchi"])):
        b, i, j, k, f, code = (int(x) for x in r)
        payload = tuple(float(x) for x in pay) + (0.0, 0.0) if 401 <= code <= 403 else ()
        rows.append((b, i, j, k, f, code, payload))
        n1, n2 = int(nc[0]), int(nc[1])
        if code == 102:
            d = [tuple(int(x) for x in donor[s]) + (float(weight[s]),) for s in range(off, off + n1 + n2)]
            chim[n] = (d[:n1], d[n1:])
        off += n1 + n2
    case = Case(f"doisneau_chimera_{closure}", nodes, [fam], num, rows)
    case.chimera = chim
    states = []
    for nd in nodes:
        st = empty_state(tuple(s - 1 for s in nd.shape[:3]), fam.nc)
        st[2:-2, 2:-2, 2:-2, :] = 1e-20
        states.append([st])
    case.state = states
    return case


# ------------------------------------------------------------ config 2
def jets_2d(n=1024, steps=500, seed=2, length=0.1, precision=0):
    """2-D single block n x n, MK and IG families advanced together (one run, two families),
    one-way coupled to a frozen gas: velocity = 32 seeded divergence-free Fourier modes
    (|k| in 1..8, RMS 10 m/s), T = 300 K, p = 101325 Pa (rho = p/(R T)). Two jets enter the
    left face at +30 and -30 deg (402: 20 um, 300 K, 10 m/s, volume fraction 1e-4); the rest
    of the left face is symmetry, the other faces extrapolation. Drag Schiller-Naumann, heat
    Ranz-Marshall; Rusanov, van Leer, SSP-RK2."""
    rng = np.random.default_rng(seed)
    dx = length / n
    nodes = box_nodes(n, n, 1, size=(length, length, dx))
    rho_m, rp, vf, speed = 1000.0, 20e-6, 1e-4, 10.0
    fams = [Family("MK", riemann="Rusanov", rho_al=rho_m, cs_al=4180.0, lv_al=2.26e6),
            Family("IG", riemann="Rusanov", rho_al=rho_m, cs_al=4180.0, lv_al=2.26e6)]
    num = Numerics(scheme="RK2", cfl=0.5, limiter="vanleer", coupled=True, drag="Schiller-Naumann",
                   heat="Ranz-Marshall", itermax=steps, precision=precision)
    j1 = (int(0.30 * n) - n // 40, int(0.30 * n) + n // 40)
    j2 = (int(0.70 * n) - n // 40, int(0.70 * n) + n // 40)
    cos30 = math.cos(PI / 6.0)
    rows = []
    for row in box_bc(1, (n, n, 1), {1: 300, 2: 400, 3: 400, 4: 400, 5: 0, 6: 0}):
        b, i, j, k, f, code, pay = row
        if f == 1 and (j1[0] <= j <= j1[1] or j2[0] <= j <= j2[1]):
            alpha = PI / 6.0 if j <= n // 2 else -PI / 6.0
            rows.append((b, i, j, k, f, 402, (vf * rho_m * speed * cos30, speed, alpha, 0.0, 300.0, rp, 0.0, 0.0)))
        else:
            rows.append(row)
    case = Case("jets_2d", [nodes], fams, num, rows)
    u, v, w = fourier_velocity(rng, (1, n, n), (dx, dx, dx), np.zeros(3), rms=10.0, ndim=2, length=length)
    T = 300.0
    rho_g = 101325.0 / (287.05 * T)
    case.gas = [_gas_layout(case, 0, rho_g, u, v, 0.0 * w, T)]
    mp = particle_mass(rp, rho_m)
    states = []
    for fam in fams:
        st = empty_state((n, n, 1), fam.nc)
        I = st[2:-2, 2:-2, 2:-2]
        I[...] = 0.0
        I[..., 0] = 1e-20
        I[..., fam.nc - 2] = 300.0
        I[..., fam.nc - 1] = 1e-20 / mp
        if fam.closure == "IG":
            I[..., 4] = 1e-20
        states.append(st)
    case.state = [states]
    return case


# --------------------------------------- the reference's published benchmark, restated
def taylor_green_ig(n=192, steps=100, h=1e-3, precision=0):
    """A case built like the reference's published performance benchmark (192^3 cube, one block, one IG
    family, a frozen Taylor-Green gas, drag and heat, no evaporation; MUSCL van Leer, Rusanov, SSP-RK2,
    CFL 0.5): cells of 1 mm; particles of 10 um and material density 1000 with bulk density
    1e-3 (1 + 0.3 cos kx cos ky cos kz), velocity (10, 7, 4) m/s, dispersion 1 m/s, 300 K; gas 1.2 kg/m3,
    u = sin kx cos ky cos kz, v = -cos kx sin ky cos kz, w = 0 (m/s), 300 K, k = 2 pi / L. Every face is
    an outflow (400)."""
    L = n * h
    nodes = box_nodes(n, n, n, size=(L, L, L))
    fam = Family("IG", riemann="Rusanov", rho_al=1000.0, cs_al=4180.0, lv_al=2.26e6)
    num = Numerics(scheme="RK2", cfl=0.5, limiter="vanleer", coupled=True, drag="Schiller-Naumann",
                   heat="Ranz-Marshall", itermax=steps, precision=precision)
    rows = box_bc(1, (n, n, n), {1: 400, 2: 400, 3: 400, 4: 400, 5: 400, 6: 400})
    case = Case("taylor_green_ig", [nodes], [fam], num, rows)
    xc = (np.arange(n) + 0.5) * h
    kk = 2.0 * PI / L
    cz, cy, cx = np.meshgrid(np.cos(kk * xc), np.cos(kk * xc), np.cos(kk * xc), indexing="ij")
    sz, sy, sx = np.meshgrid(np.sin(kk * xc), np.sin(kk * xc), np.sin(kk * xc), indexing="ij")
    rho = 1e-3 * (1.0 + 0.3 * cx * cy * cz)
    mp = particle_mass(10e-6, fam.rho_al)
    st = empty_state((n, n, n), fam.nc)
    I = st[2:-2, 2:-2, 2:-2]
    I[..., 0] = rho; I[..., 1] = 10.0; I[..., 2] = 7.0; I[..., 3] = 4.0
    I[..., 4] = rho * 1.0 / 3.0; I[..., 5] = 300.0; I[..., 6] = rho / mp
    case.state = [[st]]
    case.gas = [_gas_layout(case, 0, np.full((n, n, n), 1.2), sx * cy * cz, -cx * sy * cz, 0.0 * cx,
                            np.full((n, n, n), 300.0))]
    return case


# ------------------------------------------------------------ config 3
def droplet_material(**kw):
    d = dict(rho_al=1000.0, cs_al=4180.0, lv_al=2.26e6, emiss=0.9, evap="CEM", intf="LK", Mv=18.015,
             cpv=1996.0, Le=1.0, Yinf=0.0, Tboil=373.15, alphaE=1.0)
    d.update(kw)
    return d


def _cloud_state(rng, fam, shape, spacing, lo, L, u, v, w, median=30e-6, sigma=0.4, vf=1e-4, nblobs=16,
                 empty_rho=1e-12):
    blob, which = gaussian_blobs(rng, shape, spacing, lo, nblobs, width=0.08 * L, length=L)
    radii = median * np.exp(sigma * rng.normal(size=nblobs))
    rp = np.where(which >= 0, radii[np.maximum(which, 0)], median)
    rho = np.maximum(vf * fam.rho_al * blob, empty_rho)
    mp = 4.0 / 3.0 * PI * rp ** 3 * fam.rho_al
    nk, nj, ni = shape
    st = empty_state((ni, nj, nk), fam.nc)
    I = st[2:-2, 2:-2, 2:-2]
    I[..., 0] = rho; I[..., 1] = u; I[..., 2] = v; I[..., 3] = w
    if fam.closure == "IG":
        I[..., 4] = rho * 1e-2
    elif fam.closure == "AG":
        I[..., 4:10] = 0.0
        I[..., 4] = rho * 1e-2; I[..., 7] = rho * 1e-2; I[..., 9] = rho * 1e-2
    I[..., fam.nc - 2] = 300.0
    I[..., fam.nc - 1] = rho / mp
    return st


def gas_recipe(rng, shape, spacing, lo, L, rms=15.0):
    u, v, w = fourier_velocity(rng, shape, spacing, lo, rms=rms, ndim=3, length=L)
    blobT, _ = gaussian_blobs(rng, shape, spacing, lo, 8, width=0.15 * L, length=L)
    T = 300.0 + 1200.0 * blobT / max(float(blobT.max()), 1e-30)
    rho_g = 101325.0 / (287.05 * T)
    return rho_g, u, v, w, T


def cloud_3d(n=192, steps=200, seed=3, length=0.0192, precision=0):
    """3-D single block n^3, one AG family of water droplets (lognormal radius, median 30 um,
    sigma 0.4, volume fraction 1e-4 in 16 seeded Gaussian blobs), frozen gas of 15 m/s RMS
    Fourier velocity and 300-1500 K smooth temperature blobs. Drag, heat, grey-body radiation,
    evaporation (CEM gas side, Langmuir-Knudsen interface, MHB98 Stefan blowing). MUSCL van
    Leer with the Jameson sensor, SSP-RK3. The reference refuses Saurel for AG: Rusanov."""
    rng = np.random.default_rng(seed)
    dx = length / n
    nodes = box_nodes(n, n, n, size=(length, length, length))
    fam = Family("AG", riemann="Rusanov", **droplet_material())
    num = Numerics(scheme="RK3", cfl=0.5, limiter="vanleer", shock_detector=True, coupled=True,
                   drag="Schiller-Naumann", heat="Ranz-Marshall", blowing=True, itermax=steps, precision=precision)
    rows = box_bc(1, (n, n, n), {f: 400 for f in range(1, 7)})
    case = Case("cloud_3d", [nodes], [fam], num, rows)
    shape = (n, n, n)
    sp = (dx, dx, dx)
    rho_g, u, v, w, T = gas_recipe(rng, shape, sp, np.zeros(3), length)
    case.gas = [_gas_layout(case, 0, rho_g, u, v, w, T)]
    case.state = [[_cloud_state(rng, fam, shape, sp, np.zeros(3), length, u, v, w)]]
    return case


# ------------------------------------------------------------ config 4 / 5
def solid_material(**kw):
    d = dict(rho_al=2700.0, cs_al=900.0, lv_al=1.08e7, emiss=0.8, evap="none")
    d.update(kw)
    return d


FAMILY_RADIUS = {"MK": 10e-6, "IG": 30e-6, "AG": 60e-6}


def tree_blocks(nblocks, seed, lo=16, hi=160):
    """A tree of blocks joined face to face: block 0 first, each next block attached to a free face
    of an earlier one, its two axes along the face those of the face, the third drawn uniformly in
    lo..hi. Returns (dims, origins in cells, connections [(parent, face, child, child_face)])."""
    rng = np.random.default_rng(seed)
    dims = [tuple(int(x) for x in rng.integers(lo, hi + 1, size=3))]
    orig = [np.zeros(3, dtype=np.int64)]
    used = [set()]
    conns = []
    while len(dims) < nblocks:
        p = int(rng.integers(0, len(dims)))
        free = [f for f in range(1, 7) if f not in used[p]]
        if not free:
            continue
        f = int(rng.choice(free))
        d = (f - 1) // 2
        nd = list(dims[p])
        nd[d] = int(rng.integers(lo, hi + 1))
        fc = f + 1 if f % 2 == 1 else f - 1          # the child's face against the parent
        o = orig[p].copy()
        if f % 2 == 0:
            o[d] += dims[p][d]
        else:
            o[d] -= nd[d]
        dims.append(tuple(nd)); orig.append(o); used.append({fc})
        used[p].add(f)
        conns.append((p, f, len(dims) - 1, fc))
    return dims, orig, conns


def multiblock_tree(nblocks=48, seed=9, lo=16, hi=160, h=1e-4, families=("MK", "IG", "AG"), steps=100,
                    precision=0, evaporation_everywhere=False, scheme="RK3", gas_seed=None):
    """3-D multi-block case: nblocks blocks of U[lo, hi] cells per axis joined by matched face
    connections (101) in a seeded tree; the other faces extrapolation (400). Families MK (inert solid
    particles, 10 um), IG (water droplets, 30 um), AG (water droplets, 60 um); the gas recipe and the
    exchange terms of the 192^3 case (drag, heat, radiation, evaporation with LK and blowing). The
    per-family default Riemann solver (Saurel MK, Rusanov IG/AG), MUSCL van Leer with the Jameson
    sensor, SSP-RK3."""
    dims, orig, conns = tree_blocks(nblocks, seed, lo, hi)
    nodes = [box_nodes(*dm, lo=tuple(o * h), size=tuple(np.array(dm) * h)) for dm, o in zip(dims, orig)]
    fams = []
    for cl in families:
        mat = solid_material() if cl == "MK" else droplet_material()
        fams.append(Family(cl, **mat))
    num = Numerics(scheme=scheme, cfl=0.5, limiter="vanleer", shock_detector=True, coupled=True,
                   drag="Schiller-Naumann", heat="Ranz-Marshall", blowing=True, itermax=steps, precision=precision)
    link = {}
    for (p, f, c, fc) in conns:
        link[(p, f)] = (c, fc)
        link[(c, fc)] = (p, f)
    rows = []
    for b, (ni, nj, nk) in enumerate(dims):
        codes = {f: (101 if (b, f) in link else 400) for f in range(1, 7)}
        for row in box_bc(b + 1, (ni, nj, nk), codes):
            bb, i, j, k, f, code, pay = row
            if code == 101:
                ob, of = link[(b, f)]
                d = (f - 1) // 2
                src = [i, j, k]
                src[d] = 1 if f % 2 == 0 else dims[ob][d]     # the first cell of the block across
                rows.append((bb, i, j, k, f, 101, (ob + 1, src[0], src[1], src[2], of)))
            else:
                rows.append(row)
    case = Case(f"multiblock_{nblocks}", nodes, fams, num, rows)
    rng = np.random.default_rng(seed if gas_seed is None else gas_seed)
    ext_lo = np.min([o for o in orig], axis=0) * h
    ext_hi = np.max([o + np.array(dm) for o, dm in zip(orig, dims)], axis=0) * h
    L = float(np.max(ext_hi - ext_lo))
    # the gas recipe evaluated at every block's own cell centres, in one frame
    modes = _draw_modes(rng, 32, 1, 8)
    tblobs = [(ext_lo + rng.uniform(0.15, 0.85, size=3) * (ext_hi - ext_lo)) for _ in range(8)]
    dblobs = [(ext_lo + rng.uniform(0.15, 0.85, size=3) * (ext_hi - ext_lo)) for _ in range(16)]
    radii = {cl: FAMILY_RADIUS[cl] * np.exp(0.4 * rng.normal(size=16)) for cl in families}
    case.gas, case.state = [], []
    for b, (dm, o) in enumerate(zip(dims, orig)):
        xc = [(o[a] + np.arange(dm[a]) + 0.5) * h for a in range(3)]
        u, v, w = _eval_modes(modes, xc, L, rms=15.0)
        T = 300.0 + 1200.0 * np.minimum(_eval_blobs(tblobs, xc, 0.15 * L), 1.0)
        rho_g = 101325.0 / (287.05 * T)
        case.gas.append(_gas_layout(case, b, rho_g, u, v, w, T))
        blob = np.minimum(_eval_blobs(dblobs, xc, 0.08 * L), 1.0)
        per_fam = []
        for fam in fams:
            rp = radii[fam.closure][np.argmax(np.stack([_eval_blobs([c], xc, 0.08 * L) for c in dblobs]), axis=0)]
            floor = 1e-4 * fam.rho_al * 1e-3 if evaporation_everywhere else 1e-12
            rho = np.maximum(1e-4 * fam.rho_al * blob, floor)
            mp = 4.0 / 3.0 * PI * rp ** 3 * fam.rho_al
            st = empty_state(dm, fam.nc)
            I = st[2:-2, 2:-2, 2:-2]
            I[..., 0] = rho; I[..., 1] = u; I[..., 2] = v; I[..., 3] = w
            if fam.closure == "IG":
                I[..., 4] = rho * 1e-2
            elif fam.closure == "AG":
                I[..., 4:10] = 0.0
                I[..., 4] = rho * 1e-2; I[..., 7] = rho * 1e-2; I[..., 9] = rho * 1e-2
            I[..., fam.nc - 2] = 300.0
            I[..., fam.nc - 1] = rho / mp
            per_fam.append(st)
        case.state.append(per_fam)
    case.conns = conns
    return case


def _draw_modes(rng, nmodes, kmin, kmax):
    modes = []
    while len(modes) < nmodes:
        kv = rng.integers(-kmax, kmax + 1, size=3)
        kn = float(np.linalg.norm(kv))
        if kn < kmin or kn > kmax:
            continue
        a = rng.normal(size=3)
        a = a - kv * (a @ kv) / (kn * kn)
        modes.append((kv, a / max(np.linalg.norm(a), 1e-30) / kn, rng.uniform(0, 2 * PI)))
    return modes


def _eval_modes(modes, xc, L, rms):
    x, y, z = xc
    shape = (len(z), len(y), len(x))
    u = np.zeros(shape); v = np.zeros(shape); w = np.zeros(shape)
    for kv, a, ph in modes:
        cs = np.cos((2 * PI / L) * (kv[0] * x[None, None, :] + kv[1] * y[None, :, None] + kv[2] * z[:, None, None]) + ph)
        u += a[0] * cs; v += a[1] * cs; w += a[2] * cs
    # the RMS of the mode sum over a periodic box of side L, independent of the block
    s = rms / math.sqrt(sum(0.5 * float(a @ a) for _, a, _ in modes))
    return u * s, v * s, w * s


def _eval_blobs(centres, xc, width):
    x, y, z = xc
    out = 0.0
    for c in centres:
        out = out + (np.exp(-((x[None, None, :] - c[0]) ** 2) / (2 * width ** 2))
                     * np.exp(-((y[None, :, None] - c[1]) ** 2) / (2 * width ** 2))
                     * np.exp(-((z[:, None, None] - c[2]) ** 2) / (2 * width ** 2)))
    return out


def near_singular_ag_cloud(n=16, steps=20, corr=1.0 - 1e-9, precision=0):
    """An AG cloud whose velocity covariance is nearly singular: a Gaussian blob of bulk density
    (1e-3 kg/m3 at the centre over a floor of 1e-6 of it) moving at (3, 2, 1) m/s, every cell with the
    covariance rho theta M, theta = 0.01 m2/s2 and M = [[1, c, c], [c, 1, c], [c, c, 1]], c = corr
    (smallest eigenvalue 1 - c). Single precision rounds c to 1, so fluxes evaluated in it can carry a
    cell's covariance across the positive-definite bound. One n^3 block of 1 mm cells, extrapolation on
    every face, no gas; MUSCL van Leer, Rusanov, SSP-RK3, CFL 0.5, 60 um droplets."""
    h = 1e-3
    nodes = box_nodes(n, n, n, size=(n * h, n * h, n * h))
    fam = Family("AG", riemann="Rusanov", **droplet_material())
    num = Numerics(scheme="RK3", cfl=0.5, dt_max=1.0, limiter="vanleer", itermax=steps, precision=precision)
    xc = (np.arange(n) + 0.5) * h
    X, Y, Z = np.meshgrid(xc, xc, xc, indexing="ij")
    c0 = n * h / 2
    rho = 1e-3 * (1e-6 + np.exp(-((X - c0) ** 2 + (Y - c0) ** 2 + (Z - c0) ** 2) / (0.2 * n * h) ** 2))
    th = 0.01
    mass = particle_mass(60e-6, fam.rho_al)
    prims = [rho, 3.0, 2.0, 1.0, rho * th, rho * th * corr, rho * th * corr, rho * th, rho * th * corr,
             rho * th, 300.0, rho / mass]
    return _single_block("near_singular_ag", nodes, fam, num, {f: 400 for f in range(1, 7)}, prims)
