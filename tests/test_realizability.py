"""The FP32-flux form's realizability correction of AG states (FP64, after each update): single-precision
fluxes must not carry the velocity covariance of an occupied cell (density above rho_empty) out of the
positive-definite set by a rounding.

- FP32-induced: on a cloud whose covariance is nearly singular (smallest correlation eigenvalue 1e-9,
  which single precision rounds to 0) the plain FP64 form keeps every occupied cell positive definite,
  while the single-precision fluxes without the correction carry cells across the bound. With the
  correction it fires and no occupied cell is left outside.
- The plain form's own cases: the reference's scheme itself (the plain form, bit for bit the oracle)
  leaves some occupied AG cells of the evaporating cloud and of the multi-block tree with a covariance
  that is not positive definite in their first steps, by far more than a rounding. The correction
  leaves those as the reference leaves them: at every step the chosen form has no more such cells than
  the plain form, and it stays within 1e-4 relative L1 of the plain form in bulk density, number
  density and particle mass.
The plain form never runs the correction (the reference applies its floors only)."""
import numpy as np
import pytest

from ice_b200 import abi, configs
from ice_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from ice_b200 import build
    build.build()
    return abi.load_gpu()


def min_correlation_eigenvalue(state, rho_empty=1e-6):
    """The smallest eigenvalue of the correlation matrix D^-1/2 P D^-1/2 of every occupied interior cell
    (density above rho_empty; emptier cells keep the reference's dispersion cap instead)."""
    p = state[2:-2, 2:-2, 2:-2].reshape(-1, 12)
    p = p[p[:, 0] > rho_empty]
    P = np.empty((p.shape[0], 3, 3))
    P[:, 0, 0], P[:, 0, 1], P[:, 0, 2] = p[:, 4], p[:, 5], p[:, 6]
    P[:, 1, 0], P[:, 1, 1], P[:, 1, 2] = p[:, 5], p[:, 7], p[:, 8]
    P[:, 2, 0], P[:, 2, 1], P[:, 2, 2] = p[:, 6], p[:, 8], p[:, 9]
    d = 1.0 / np.sqrt(np.stack([p[:, 4], p[:, 7], p[:, 9]], axis=1))
    C = P * d[:, :, None] * d[:, None, :]
    return np.linalg.eigvalsh(C)[:, 0]


def _non_pd(solver, case, p):
    """Occupied cells whose covariance is not positive definite (beyond the FP64 rounding of the
    eigenvalue computation)."""
    return sum(int((min_correlation_eigenvalue(solver.download(b, p)) < -1e-12).sum()) for b in range(len(case.nodes)))


def _run(case, gpu, p, steps):
    s = Solver(case, gpu)
    bad = []
    for _ in range(steps):
        out = s.step(1)
        assert out.status == 0
        bad.append(_non_pd(s, case, p))
    return s, out, bad


def test_fp32_induced_violations_are_corrected(gpu):
    _, out, bad = _run(configs.near_singular_ag_cloud(precision=abi.PREC_FP64), gpu, 0, 20)
    assert sum(bad) == 0 and out.nrealized == 0
    off = configs.near_singular_ag_cloud(precision=abi.PREC_FP32FLUX)
    off.numerics.realize = False
    _, out, bad = _run(off, gpu, 0, 20)
    assert sum(bad) > 0 and out.nrealized == 0, "the single-precision fluxes never crossed the bound"
    _, out, bad = _run(configs.near_singular_ag_cloud(precision=abi.PREC_FP32FLUX), gpu, 0, 20)
    assert sum(bad) == 0 and out.nrealized > 0


@pytest.mark.parametrize("make", [
    lambda prec: configs.cloud_3d(n=32, steps=20, length=0.0032, precision=prec),
    lambda prec: configs.multiblock_tree(nblocks=6, seed=3, lo=8, hi=16, steps=20, precision=prec),
], ids=["cloud3d", "multiblock"])
def test_plain_form_cases(gpu, make):
    plain_case = make(abi.PREC_FP64)
    p = [f.closure for f in plain_case.families].index("AG")
    plain, out, bad_plain = _run(plain_case, gpu, p, 20)
    assert bad_plain[0] > 0 and out.nrealized == 0        # the scheme's own first steps
    chosen_case = make(abi.PREC_FP32FLUX)
    chosen, out, bad = _run(chosen_case, gpu, p, 20)
    assert all(x <= y for x, y in zip(bad, bad_plain)), (bad, bad_plain)
    a, b = chosen.download_all(), plain.download_all()
    for name, fn in (("rho", lambda x, nc: x[..., 0]), ("n", lambda x, nc: x[..., nc - 1]),
                     ("mass", lambda x, nc: x[..., 0] / x[..., nc - 1])):
        num = den = 0.0
        for ba, bb in zip(a, b):
            for f, xa, xb in zip(plain_case.families, ba, bb):
                ya, yb = fn(xa[2:-2, 2:-2, 2:-2], f.nc), fn(xb[2:-2, 2:-2, 2:-2], f.nc)
                num += float(np.abs(ya - yb).sum()); den += float(np.abs(yb).sum())
        assert num / den <= 1e-4, (name, num / den)
