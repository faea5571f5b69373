"""The reference's fast cases that exercise the step, on the oracle and on the CUDA path:
test/fast/inlet-direction (an inlet on a face whose normal points out of the domain injects into it),
test/fast/res-threshold (a steady run ends when its density residual has fallen by res-threshold
from the first non-zero one; Mod_Explicit.f90:193-240), the family leg of test/fast/equiv3d (a
family in company steps as it does alone), test/fast/populations (copy c of the boundary table
drives family c) and the step-level legs of test/fast/restart-exact (a restart goes on as the
uninterrupted run would)."""
import numpy as np
import pytest

from ice_b200 import abi, configs
from ice_b200.case import SetupError
from ice_b200.solver import SolveError, Solver

THR, ITERS = 1e-5, 20000


def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return abi.load_gpu()


def _inlet_direction(lib):
    """normal: a 402 inlet along the normal of face 2 gives the inlet cell u = -10 m/s and the injected
    density gp / v = 0.1 after 200 steps, to 1e-9. angles: a 401 inlet at alpha = 180 deg in a gas moving
    along -x gives u = -kV 10 m/s there (inlet-direction/run.py: normal, angles)."""
    s = Solver(configs.inlet_duct("normal"), lib)
    assert s.step(200).status == 0
    p = s.download(0, 0)[2, 2, 2:-2]
    assert abs(p[-1, 1] + 10.0) <= 1e-9 * 10.0 and abs(p[-1, 0] - 0.1) <= 1e-9 * 0.1
    s = Solver(configs.inlet_duct("angles"), lib)
    assert s.step(200).status == 0
    p = s.download(0, 0)[2, 2, 2:-2]
    assert abs(p[-1, 1] + 10.0) <= 1e-9 * 10.0


def _history(lib, case):
    """The density residual of every step, one call per step, up to the step that ends the run."""
    s = Solver(case, lib)
    rows = []
    for _ in range(ITERS):
        out = s.step(1)
        assert out.status == 0 and out.have_norm == 1
        rows.append((out.iter, out.residual[0]))
        if out.todo == 3:
            break
    ref = np.zeros(1)
    assert lib.get_res_reference(s.ctx, abi.ptr(ref)) == abi.OK
    return rows, float(ref[0])


def _ended_on_residual(rows, ref):
    """The last row is the first after the first non-zero residual at or below THR times it."""
    k0 = next(k for k, (_, r) in enumerate(rows) if r > 0.0)
    assert ref == rows[k0][1]
    below = [k for k, (_, r) in enumerate(rows) if k > k0 and r <= THR * ref]
    return bool(below) and below[0] == len(rows) - 1


def _res_threshold(lib):
    """scaling: a density wave carried out of a 1-D stream, at loading 1 and 2^-16 (an exact scaling of
    the MK equations): both end on their first residual below 1e-5 of their first, at the same
    iteration, and one call of 20000 steps ends at that step. at rest: the first one-stage step moves no
    mass, its residual is exactly zero and ends nothing. frozen: every residual is zero, the run goes to
    its 40 iterations (res-threshold/run.py)."""
    ends = []
    for scale in (1.0, 2.0 ** -16):
        rows, ref = _history(lib, configs.stream_tube("scaling", scale))
        assert _ended_on_residual(rows, ref)
        ends.append(rows[-1][0])
        out = Solver(configs.stream_tube("scaling", scale), lib).step(ITERS)
        assert out.todo == 3 and out.iter == rows[-1][0]
    assert ends[0] == ends[1] and 1 < ends[0] < ITERS
    rows, ref = _history(lib, configs.stream_tube("at_rest"))
    assert rows[0][1] == 0.0 and len(rows) > 1 and _ended_on_residual(rows, ref) and rows[-1][0] < ITERS
    s = Solver(configs.stream_tube("frozen"), lib)
    out = s.step(40)
    assert out.iter == 40 and out.todo == 3 and out.residual[0] == 0.0
    ref = np.zeros(1)
    assert lib.get_res_reference(s.ctx, abi.ptr(ref)) == abi.OK and ref[0] == 0.0


def _family_company(lib, precision=0):
    """The MK + IG + AG multi-block case (8 blocks joined by connections, drag, heat, radiation and
    evaporation) against each family run alone: within a step the families are independent, and with
    dt-max binding every cell the step is the same, so family K in company equals family K alone value
    for value (equiv3d/run.py, family leg)."""
    def make(solo=None):
        c = configs.multiblock_tree(nblocks=8, seed=3, lo=5, hi=11, steps=6, precision=precision)
        c.numerics.dt_max = 1e-9
        if solo is not None:
            c.families = [c.families[solo]]
            c.state = [[per_fam[solo]] for per_fam in c.state]
        return c
    case = make()
    s = Solver(case, lib)
    out = s.step(6)
    assert out.status == 0 and out.dtglobal == 1e-9
    for k in range(3):
        alone = Solver(make(k), lib)
        assert alone.step(6).status == 0
        for b in range(len(case.nodes)):
            assert np.array_equal(alone.download(b, 0)[2:-2, 2:-2, 2:-2], s.download(b, k)[2:-2, 2:-2, 2:-2]), (k, b)


def _populations(lib):
    """proportional: three copies of the table whose inlet mass fluxes are 1, 2 and 4 times the first,
    and loadings scaled alike: family p is 2^(p-1) times family 1 in density and number density and
    equal in velocity and temperature, to 1e-12 of each field, as are its density residual (scaled) and
    its velocity and temperature residuals; the domain's norms are the roots of the sums of the
    families' squares. shared: one copy, three families: the families are identical. mismatch: two
    copies for three families stop the set-up (populations/run.py)."""
    rel = lambda a, b: float(np.abs(a - b).max()) / max(float(np.abs(b).max()), 1e-300)
    s = Solver(configs.population_duct(3, 3, True), lib)
    assert s.step(30).status == 0
    f = [s.download(0, p)[2:-2, 2:-2, 2:-2] for p in range(3)]
    assert float(f[0][..., 0].max()) > 1e-3
    for p in (1, 2):
        for v in (0, 5):
            assert rel(f[p][..., v], 2.0 ** p * f[0][..., v]) <= 1e-12
        for v in (1, 2, 3, 4):
            assert rel(f[p][..., v], f[0][..., v]) <= 1e-12
    tot, fam = np.zeros(5), np.zeros(15)
    assert lib.residual_norm(s.ctx, abi.ptr(tot), abi.ptr(fam)) == abi.OK
    fam = fam.reshape(3, 5)
    for p in (1, 2):
        assert abs(fam[p, 0] / (2.0 ** p * fam[0, 0]) - 1.0) <= 1e-12
        assert np.all(np.abs(fam[p, 1:] - fam[0, 1:]) <= 1e-12 * np.abs(fam[0, 1:]).max())
    assert np.all(np.abs(tot - np.sqrt((fam ** 2).sum(0))) <= 1e-12 * np.abs(tot).max())
    s = Solver(configs.population_duct(1, 3, False), lib)
    assert s.step(30).status == 0
    f = [s.download(0, p)[2:-2, 2:-2, 2:-2] for p in range(3)]
    assert np.array_equal(f[1], f[0]) and np.array_equal(f[2], f[0])
    with pytest.raises(SetupError, match="copies of the boundary table"):
        Solver(configs.population_duct(2, 3, False), lib)


def _restart(lib, make, n, total):
    """Run A: `total` steps in one call. Run B: n steps, its state, time, iteration and residual reference
    taken into a new context, then the rest. Returns both final reports and states."""
    a = Solver(make(), lib)
    oa = a.step(total)
    b = Solver(make(), lib)
    ob = b.step(n)
    mid = b.download_all()
    ref = np.zeros(1)
    assert lib.get_res_reference(b.ctx, abi.ptr(ref)) == abi.OK
    c = Solver(make(), lib, upload=False)
    c.upload(mid)
    c.set_time(ob.time, ob.iter, ob.iter)
    assert lib.set_res_reference(c.ctx, float(ref[0])) == abi.OK
    oc = c.step(total - n)
    return oa, oc, a.download_all(), c.download_all()


def _restart_checks(lib):
    """res-threshold: a steady stream that res-threshold stops at iteration 444; restarted at 200, with
    its residual reference carried over, it stops at 444 too, in the same state. wedge: the one-degree
    wedge of Axis/AG with its cloud moving along x at 1 m/s (w, P13 and P23 frozen), 40 = 20 + 20 steps.
    families: the populations duct, copy c driving family c, 30 = 15 + 15 steps. Every state equal bit
    for bit (restart-exact/run.py)."""
    oa, oc, ra, rc = _restart(lib, lambda: configs.stream_tube("scaling"), 200, ITERS)
    assert 200 < oa.iter == oc.iter < ITERS and oa.todo == oc.todo == 3

    def wedge():
        c = configs.axis_wedge("AG")
        c.numerics.itermax = 40
        c.state[0][0][2:-2, 2:-2, 2:-2, 1] = 1.0
        return c
    cases = [(ra, rc), _restart(lib, wedge, 20, 40)[2:], _restart(lib, lambda: configs.population_duct(3, 3, True),
                                                               15, 30)[2:]]
    for a, c in cases:
        for per_a, per_c in zip(a, c):
            for x, y in zip(per_a, per_c):
                assert np.array_equal(x[2:-2, 2:-2, 2:-2], y[2:-2, 2:-2, 2:-2])


def test_restart_oracle(orc):
    _restart_checks(orc)


def test_populations_oracle(orc):
    _populations(orc)


def _gas_refusals(lib):
    """refusals (test/fast/refusals: inlet 401 and 403 without a gas). As read_bc (IO_BC.f90:264-271)
    does while it reads the table, set_records refuses a 401 or 403 inlet with a non-zero mass flux in
    a run without a gas phase; the same inlet with a zero mass flux mirrors (Lib_Ghost.f90:409), reads
    no gas and is accepted. A coupled run whose gas is missing in a block is refused by the step
    before any launch. Both libraries refuse at the same call with the same reason."""
    for code in (401, 403):
        case = configs.inlet_duct("angles")
        case.gas = []
        case.numerics.coupled = False
        case.build_geometry()
        case.build_records(lib)
        rows = case.rec_int[:, 5] == 401
        assert rows.any()
        case.rec_int[rows, 5] = code
        with pytest.raises(SolveError, match="set_records.*takes its speed from the gas"):
            Solver(case, lib)
        case.rec_real[rows, 0] = 0.0                 # a zero-flux inlet reads no gas: accepted
        s = Solver(case, lib)
        out = s.step(3)
        assert out.status == 0 and out.iter == 3
        assert np.isfinite(s.download(0, 0)[2:-2, 2:-2, 2:-2]).all()
    case = configs.multiblock_tree(nblocks=3, seed=2, lo=4, hi=6, steps=2)
    case.gas = case.gas[:1]
    s = Solver(case, lib)
    with pytest.raises(SolveError, match="step failed.*gas of every block"):
        s.step(1)


def test_gas_refusals_oracle(orc):
    _gas_refusals(orc)


def test_thread_count_equivalence_oracle(orc):
    """equiv3d's threads leg (and openmp-equiv): a 12-block, three-family case steps to the same bits on
    1, 2, 3, 4 and 8 threads. The oracle computes each face flux once and sums a cell's boundary
    records in face order, as the reference's owner-computes loops do, so no sum depends on the
    schedule."""
    runs = []
    before = orc.set_threads(0)                 # 0 reads the count and changes nothing
    try:
        for nt in (1, 2, 3, 4, 8):
            orc.set_threads(nt)
            s = Solver(configs.multiblock_tree(nblocks=12, seed=1, lo=6, hi=10, steps=4), orc)
            assert s.step(4).status == 0
            runs.append(s.download_all())
    finally:
        orc.set_threads(before)
    for r in runs[1:]:
        for pa, pb in zip(runs[0], r):
            for a, b in zip(pa, pb):
                assert np.array_equal(a[2:-2, 2:-2, 2:-2], b[2:-2, 2:-2, 2:-2])


def test_family_company_oracle(orc):
    _family_company(orc)


def test_inlet_direction_oracle(orc):
    _inlet_direction(orc)


def test_res_threshold_oracle(orc):
    _res_threshold(orc)


def test_res_reference_is_settable(orc):
    """A restart gives the run its reference back: with one larger than any residual of the run, the
    first step ends it."""
    s = Solver(configs.stream_tube("scaling"), orc)
    assert orc.set_res_reference(s.ctx, 1e30) == abi.OK
    out = s.step(ITERS)
    assert out.iter == 1 and out.todo == 3


@pytest.mark.gpu
def test_inlet_direction_gpu():
    _inlet_direction(_gpu())


@pytest.mark.gpu
def test_res_threshold_gpu():
    _res_threshold(_gpu())


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_FP32FLUX], ids=["fp64", "fp32flux"])
def test_family_company_gpu(precision):
    _family_company(_gpu(), precision)


@pytest.mark.gpu
def test_populations_gpu():
    _populations(_gpu())


@pytest.mark.gpu
def test_restart_gpu():
    _restart_checks(_gpu())


@pytest.mark.gpu
def test_gas_refusals_gpu():
    _gas_refusals(_gpu())
