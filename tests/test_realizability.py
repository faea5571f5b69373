"""The FP32-flux form's realizability correction of AG states (FP64, after each update): the velocity
covariance stays positive definite. On a cloud whose covariance is nearly singular (smallest
correlation eigenvalue 1e-9, which single precision rounds to 0) the single-precision fluxes carry
cells across the bound, and the correction fires and restores positive definiteness in every cell. The
plain form never runs it (the reference applies its floors only), and on the plain form's parity cases
the chosen form's correction never fires."""
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


def min_correlation_eigenvalue(state):
    """The smallest eigenvalue of every interior cell's correlation matrix D^-1/2 P D^-1/2."""
    p = state[2:-2, 2:-2, 2:-2].reshape(-1, 12)
    P = np.empty((p.shape[0], 3, 3))
    P[:, 0, 0], P[:, 0, 1], P[:, 0, 2] = p[:, 4], p[:, 5], p[:, 6]
    P[:, 1, 0], P[:, 1, 1], P[:, 1, 2] = p[:, 5], p[:, 7], p[:, 8]
    P[:, 2, 0], P[:, 2, 1], P[:, 2, 2] = p[:, 6], p[:, 8], p[:, 9]
    d = 1.0 / np.sqrt(np.stack([p[:, 4], p[:, 7], p[:, 9]], axis=1))
    C = P * d[:, :, None] * d[:, None, :]
    return np.linalg.eigvalsh(C)[:, 0]


def test_correction_restores_positive_definiteness(gpu):
    s = Solver(configs.near_singular_ag_cloud(precision=abi.PREC_FP32FLUX), gpu)
    fired = 0
    for _ in range(20):
        out = s.step(1)
        assert out.status == 0
        fired = out.nrealized
        assert min_correlation_eigenvalue(s.download(0, 0)).min() > 0.0
    assert fired > 0, "the single-precision fluxes never crossed the bound: the case tests nothing"
    plain = Solver(configs.near_singular_ag_cloud(precision=abi.PREC_FP64), gpu)
    out = plain.step(20)
    assert out.status == 0 and out.nrealized == 0


@pytest.mark.parametrize("make", [
    lambda: configs.cloud_3d(n=32, steps=20, length=0.0032, precision=abi.PREC_FP32FLUX),
    lambda: configs.multiblock_tree(nblocks=6, seed=3, lo=8, hi=16, steps=20, precision=abi.PREC_FP32FLUX),
], ids=["cloud3d", "multiblock"])
def test_correction_never_fires_on_resolved_cases(gpu, make):
    case = make()
    out = Solver(case, gpu).step(case.numerics.itermax)
    assert out.status == 0 and out.nrealized == 0
