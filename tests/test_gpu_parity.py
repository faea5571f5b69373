"""Parity of the CUDA solve stage (plain FP64 form) with the CPU oracle, through the C ABI.

The bar (the reference's own FP64 CPU path, restated by the oracle): 1e-12 relative L-infinity
per field after the stated step count, and bit-exact block connectivity and index maps. Where no
transcendental function enters (no sources, no sensor) the two are bit-identical, and the tests
say so by asserting equality.
"""
import numpy as np
import pytest

from ice_b200 import abi, configs
from ice_b200.solver import Solver

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def gpu():
    from ice_b200 import build
    build.build()
    return abi.load_gpu()


def groups(nc):
    g = [[0], [1, 2, 3]]
    if nc == 12:
        g.append([4, 5, 6, 7, 8, 9])
        g += [[10], [11]]
    else:
        g += [[v] for v in range(4, nc)]
    return g


def compare(sg, so, case, exact=False):
    """Largest error of any field relative to the largest value of its group, over every block and
    family (interior cells)."""
    worst = 0.0
    for p, fam in enumerate(case.families):
        ga = [sg.download(b, p)[2:-2, 2:-2, 2:-2] for b in range(len(case.nodes))]
        oa = [so.download(b, p)[2:-2, 2:-2, 2:-2] for b in range(len(case.nodes))]
        for grp in groups(fam.nc):
            scale = max(max(float(np.abs(o[..., grp]).max()) for o in oa), 1e-300)
            for v in grp:
                err = max(float(np.abs(g[..., v] - o[..., v]).max()) for g, o in zip(ga, oa))
                worst = max(worst, err / scale)
                if exact:
                    for g, o in zip(ga, oa):
                        assert np.array_equal(g[..., v], o[..., v]), (p, v, float(np.abs(g[..., v] - o[..., v]).max()))
    return worst


def run_pair(gpu, orc, make, steps, exact=False, chunks=1):
    cg, co = make(), make()
    sg, so = Solver(cg, gpu), Solver(co, orc)
    for _ in range(chunks):
        og = sg.step(steps // chunks)
        oo = so.step(steps // chunks)
    assert og.status == 0 and oo.status == 0
    assert og.iter == oo.iter == steps
    if exact:
        assert og.time == oo.time and og.dtglobal == oo.dtglobal
    else:
        assert abs(og.time - oo.time) <= TOL * abs(oo.time)
    err = compare(sg, so, cg, exact=exact)
    assert err <= TOL, err
    return sg, so, cg


def test_riemann_1d_bit_exact(gpu, orc):
    # config 1 at its full size: 2000 cells, IG, HLLE, minmod, SSP-RK3 (200 of its 1000 steps here;
    # the full count runs in test_riemann_1d_full_steps)
    run_pair(gpu, orc, lambda: configs.riemann_1d(n=2000, steps=200), 200, exact=True)


@pytest.mark.slow
def test_riemann_1d_full_steps(gpu, orc):
    run_pair(gpu, orc, lambda: configs.riemann_1d(n=2000, steps=1000), 1000, exact=True)


@pytest.mark.parametrize("closure", ["MK", "IG", "AG"])
def test_crossing_jets_bit_exact(gpu, orc, closure):
    # steady (per-cell dt), inlets 402 with injected ghosts, symmetry and extrapolation faces
    run_pair(gpu, orc, lambda: configs.crossing_jets(closure, steps=300), 300, exact=True)


def test_crossing_jets_matches_reference_output(gpu):
    """The CUDA path against the field the reference's own binary wrote (5000 iterations)."""
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / "crossing_jets_IG.npz")
    s = Solver(configs.crossing_jets("IG"), gpu)
    s.step(5000)
    p = s.download(0, 0)[2, 2:-2, 2:-2]
    l2 = float(np.sqrt(np.mean((p[..., 0] - g["field"][0]) ** 2)))
    assert l2 <= 1e-12


def test_res_reference_matches_reference_output(gpu):
    """The first non-zero density residual of the crossing-jets and chimera cases against the value the
    reference's binary stored with its solutions (the oracle's pin, through the CUDA path)."""
    from pathlib import Path
    gold = Path(__file__).resolve().parent / "golden"
    g = np.load(gold / "restart_counters.npz")
    chim = dict(np.load(gold / "chimera_IG.npz"))
    cases = [(configs.crossing_jets(cl, steps=5000), float(g[f"{cl}_ICE_RES_REFERENCE"])) for cl in ("MK", "IG", "AG")]
    cases.append((configs.doisneau_chimera(chim), float(g["IG_chimera_ICE_RES_REFERENCE"])))
    for case, want in cases:
        case.numerics.res_threshold = 1e-10
        s = Solver(case, gpu)
        assert s.step(1).status == 0
        got = np.zeros(1)
        assert gpu.get_res_reference(s.ctx, abi.ptr(got)) == abi.OK
        assert abs(got[0] / want - 1.0) <= 1e-12, (got[0], want)


def _chimera(steps):
    from pathlib import Path
    g = dict(np.load(Path(__file__).resolve().parent / "golden" / "chimera_IG.npz"))
    return g, configs.doisneau_chimera(g, steps=steps)


def test_chimera_bit_exact(gpu, orc):
    # two overlapping blocks joined by chimera faces (102): ghost cells blended from donor cells
    run_pair(gpu, orc, lambda: _chimera(400)[1], 400, exact=True)


def test_chimera_matches_reference_output(gpu):
    """The CUDA path against the density the reference's own binary wrote on its chimera case."""
    g, case = _chimera(5000)
    s = Solver(case, gpu)
    s.step(5000)
    for b in range(2):
        p = s.download(b, 0)[2, 2:-2, 2:-2, 0]
        l2 = float(np.sqrt(np.mean((p - g[f"rho{b + 1}"]) ** 2)))
        assert l2 <= 1e-12, (b, l2)


def _with_imports(case, seed, scale):
    """The coupler's imports for every block and family: births into a quarter of the cells (mass at
    up to `scale` per second with a momentum of 0-30 m/s), removal from another quarter (up to a
    tenth of the local density per second)."""
    rng = np.random.default_rng(seed)
    out = []
    for b, (ni, nj, nk) in enumerate(case.dims):
        per = []
        for p, fam in enumerate(case.families):
            rho = case.state[b][p][2:-2, 2:-2, 2:-2, 0]
            imp = np.zeros((nk, nj, ni, fam.nc))
            u = rng.random((nk, nj, ni))
            born = u < 0.25
            gone = u > 0.75
            m = scale * rng.random((nk, nj, ni))
            imp[..., 0] = np.where(born, m, 0.0) - np.where(gone, 0.1 * np.nan_to_num(rho) * rng.random((nk, nj, ni)), 0.0)
            for a in range(3):
                imp[..., 1 + a] = np.where(born, m * 30.0 * (rng.random((nk, nj, ni)) - 0.5), 0.0)
            per.append(np.ascontiguousarray(imp))
        out.append(per)
    return out


def _set_imports(lib, solver, imports):
    for b, per in enumerate(imports):
        for p, imp in enumerate(per):
            assert lib.set_imports(solver.ctx, b + 1, p + 1, abi.ptr(imp)) == 0


@pytest.mark.parametrize("args", [(2, None, False, False), (2, 3, False, False), (0, 3, False, False),
                                  (2, 1, False, False), (2, 1, False, True), (0, 3, True, False)],
                         ids=["E1", "E2", "E4", "E5", "E6", "E7"])
def test_empty_tube_imports_bit_exact(gpu, orc, args):
    # the unit test's tube of empty cells that the coupler's imports fill: its steps and states
    n_occ, cell, ta, narrow = args
    res = []
    for lib in (gpu, orc):
        case = configs.empty_tube(n_occ, ta, narrow, steps=3)
        s = Solver(case, lib)
        if cell is not None:
            imp = np.zeros((1, 1, 4, 6))
            imp[0, 0, cell - 1] = [2e2, 2e2 * 800.0, 0.0, 0.0, 0.0, 0.0]
            assert lib.set_imports(s.ctx, 1, 1, abi.ptr(imp)) == 0
        out = s.step(3)
        res.append((out.status, out.dtglobal, out.time, s.download(0, 0)[2, 2, 2:-2]))
    (st_g, dt_g, t_g, p_g), (st_o, dt_o, t_o, p_o) = res
    assert st_g == st_o == 0 and dt_g == dt_o and t_g == t_o
    assert np.array_equal(p_g, p_o)


@pytest.mark.parametrize("steady", [False, True], ids=["time_accurate", "steady"])
def test_multiblock_imports(gpu, orc, steady):
    # the coupler's births and removals in every family of a multi-block case
    def make():
        c = configs.multiblock_tree(nblocks=5, seed=4, lo=5, hi=10, steps=6)
        c.numerics.time_accurate = not steady
        return c
    cg, co = make(), make()
    imports = _with_imports(cg, 11, 50.0)
    sg, so = Solver(cg, gpu), Solver(co, orc)
    _set_imports(gpu, sg, imports)
    _set_imports(orc, so, imports)
    og, oo = sg.step(6), so.step(6)
    assert og.status == 0 and oo.status == 0
    assert abs(og.dtglobal - oo.dtglobal) <= TOL * abs(oo.dtglobal)
    err = compare(sg, so, cg)
    assert err <= TOL, err


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32FLUX], ids=["fp64", "fp32flux"])
def test_exchange_rates(gpu, orc, prec):
    # two-way coupling: the rates the gas receives from every family over a step (3 RK stages). The
    # plain form against the oracle to 1e-12 of each component's largest value; the chosen form to 1e-4,
    # its single-precision fluxes and sources alone: its realizability correction off, since it moves
    # the AG cells that the scheme itself leaves with a covariance that is not positive definite in the
    # first steps of this case (tests/test_realizability.py)
    make = lambda: configs.multiblock_tree(nblocks=5, seed=4, lo=5, hi=10, steps=4, precision=prec)
    cg, co = make(), make()
    cg.numerics.precision = prec
    cg.numerics.realize = False
    co.numerics.precision = abi.PREC_FP64
    sg, so = Solver(cg, gpu), Solver(co, orc)
    assert gpu.set_exchange(sg.ctx, 1) == 0 and orc.set_exchange(so.ctx, 1) == 0
    assert sg.step(4).status == 0 and so.step(4).status == 0
    tol = TOL if prec == abi.PREC_FP64 else 1e-4
    for b, (ni, nj, nk) in enumerate(cg.dims):
        for p in range(len(cg.families)):
            xg, xo = np.zeros((nk, nj, ni, 5)), np.zeros((nk, nj, ni, 5))
            assert gpu.exchange_rate(sg.ctx, b + 1, p + 1, abi.ptr(xg)) == 0
            assert orc.exchange_rate(so.ctx, b + 1, p + 1, abi.ptr(xo)) == 0
            for m in range(5):
                scale = max(float(np.max(np.abs(xo[..., m]))), 1e-300)
                assert float(np.max(np.abs(xg[..., m] - xo[..., m]))) <= tol * scale, (b, p, m)


def _irs(case):
    case.numerics.irs = True
    case.numerics.irs_beta = 0.5
    case.numerics.time_accurate = False
    return case


def test_irs_steady_1d_bit_exact(gpu, orc):
    # implicit residual smoothing (steady runs only): the 1-D tube converges with it
    run_pair(gpu, orc, lambda: _irs(configs.riemann_1d(n=400, steps=100)), 100, exact=True)


def test_irs_2d_and_3d_bit_exact(gpu, orc):
    # both directions of the crossing jets and the three of a block tree, over the steps before
    # the smoothed residual drives an empty cell negative
    run_pair(gpu, orc, lambda: _irs(configs.crossing_jets("IG", steps=20)), 20, exact=True)
    def mb():
        c = configs.multiblock_tree(nblocks=6, seed=3, lo=6, hi=10, steps=10)
        c.numerics.coupled = False
        c.numerics.shock_detector = False
        c.gas = []
        return _irs(c)
    run_pair(gpu, orc, mb, 10, exact=True)


def test_irs_failure_at_the_same_iteration(gpu, orc):
    """Where the reference's algorithm itself breaks down (IRS spreading mass into empty cells),
    the device stops at the same iteration with the same status as the oracle."""
    make = lambda: _irs(configs.crossing_jets("IG", steps=100))
    sg, so = Solver(make(), gpu), Solver(make(), orc)
    fail_g = fail_o = None
    for n in range(1, 101):
        if fail_g is None and sg.step(1, check=False).status:
            fail_g = (n, sg.last.status)
        if fail_o is None and so.step(1, check=False).status:
            fail_o = (n, so.last.status)
        if fail_g and fail_o:
            break
    assert fail_o is not None and fail_g is not None
    assert fail_g[0] == fail_o[0] and (fail_g[1] & fail_o[1])


def test_jets_2d_coupled(gpu, orc):
    # config 2 shape (MK + IG, drag and heat, two 402 jets), reduced to 96^2 for the oracle
    run_pair(gpu, orc, lambda: configs.jets_2d(n=96, steps=40), 40)


def test_jets_2d_with_sensor(gpu, orc):
    # the Jameson sensor in a 2-D run: the stage kernel reads the ghost planes above and below
    def make():
        c = configs.jets_2d(n=64, steps=60)
        c.numerics.shock_detector = True
        return c
    run_pair(gpu, orc, make, 60)


def test_taylor_green_ig(gpu, orc):
    # the shape of the reference's published 192^3 benchmark (IG, frozen Taylor-Green gas, SSP-RK2), 32^3
    run_pair(gpu, orc, lambda: configs.taylor_green_ig(n=32, steps=40), 40)


def test_cloud_3d_evaporating_ag(gpu, orc):
    # config 3 shape (AG, Jameson sensor, drag, heat, radiation, evaporation LK + blowing), 24^3
    run_pair(gpu, orc, lambda: configs.cloud_3d(n=24, steps=12, length=0.0024), 12)


@pytest.mark.parametrize("closure", ["MK", "IG", "AG"])
def test_wedge_one_cell_deep_bit_exact(gpu, orc, closure):
    # the reference's one-degree wedge (one cell deep in k, code 200 on both k faces): each k face's
    # second ghost layer is the other face's first, so the ghost layers run as two launches. A seeded
    # perturbation of the density (5 %, one drop size) and the axial velocity makes every ghost value
    # matter. The wedge's swirl (w; with AG also P13 and P23) is frozen at set-up, as the reference does.
    steps = 40

    def make():
        case = configs.axis_wedge(closure)
        case.numerics.itermax = steps
        I = case.state[0][0][2:-2, 2:-2, 2:-2]
        rng = np.random.default_rng(5)
        mp = I[..., -1] / I[..., 0]
        I[..., 0] *= 1.0 + rng.uniform(-0.05, 0.05, I[..., 0].shape)
        I[..., 1] += rng.uniform(-0.1, 0.1, I[..., 1].shape)
        I[..., -1] = I[..., 0] * mp
        return case
    run_pair(gpu, orc, make, steps, exact=True)


def test_multiblock_three_families(gpu, orc):
    # config 4 shape: a seeded tree of blocks joined by 101 connections, MK + IG + AG
    run_pair(gpu, orc, lambda: configs.multiblock_tree(nblocks=8, seed=3, lo=5, hi=11, steps=6), 6)


def test_index_maps_bit_exact(gpu, orc):
    case = configs.multiblock_tree(nblocks=10, seed=5, lo=4, hi=9, families=("MK", "AG"), steps=1)
    sg = Solver(case, gpu, upload=False)
    so = Solver(configs.multiblock_tree(nblocks=10, seed=5, lo=4, hi=9, families=("MK", "AG"), steps=1), orc,
                upload=False)
    for p in range(2):
        a, b = sg.index_maps(p), so.index_maps(p)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_restart_exact(gpu):
    """2N steps equal N steps, a download, an upload into a new context and N more, bit for bit
    (the reference's RestartExact gate)."""
    make = lambda: configs.multiblock_tree(nblocks=5, seed=7, lo=5, hi=9, steps=10)
    a = Solver(make(), gpu)
    a.step(10)
    ref = a.download_all()
    b = Solver(make(), gpu)
    o = b.step(5)
    mid = b.download_all()
    c = Solver(make(), gpu, upload=False)
    c.upload(mid)
    c.set_time(o.time, o.iter, o.iter)
    c.step(5)
    got = c.download_all()
    for rb, gb in zip(ref, got):
        for r, g in zip(rb, gb):
            assert np.array_equal(r[2:-2, 2:-2, 2:-2], g[2:-2, 2:-2, 2:-2])


def test_residual_norm(gpu, orc):
    sg, so, case = run_pair(gpu, orc, lambda: configs.multiblock_tree(nblocks=4, seed=2, lo=5, hi=8, steps=3), 3)
    tg, fg = sg.residual_norm()
    to, fo = so.residual_norm()
    assert np.all(np.abs(tg - to) <= 1e-12 * np.maximum(np.abs(to), 1e-300))
    assert np.all(np.abs(fg - fo) <= 1e-12 * np.maximum(np.abs(fo), 1e-300))


def test_nan_state_is_reported_not_trapped(gpu):
    """A NaN planted in the state on the host ends the step with ICE_GPU_ESTATE and a status bit
    (an unphysical first-order face, where the reference's compute_flux stops with error stop 1),
    and the context stays usable."""
    case = configs.crossing_jets("IG", n=16, steps=2)
    st = case.state[0][0].copy()
    st[2, 5, 5, 0] = 0.5
    st[2, 5, 5, 1] = np.nan
    case.state = [[st]]
    s = Solver(case, gpu)
    out = s.step(1, check=False)
    assert out.status & (abi.ST_NAN_STATE | abi.ST_BAD_RECON)
    assert np.isfinite(s.download(0, 0)[2, 10, 10, 0])
