"""The chosen form (FP32 reconstruction, Riemann fluxes and sources; FP64 RK accumulation, dt and
norms) against the plain FP64 form on the device, on the same inputs: relative L1 error of bulk
density, number density and particle mass within 1e-4."""
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


def rel_l1(a, b, case):
    out = {}
    for name, fn in (("rho", lambda p, nc: p[..., 0]), ("n", lambda p, nc: p[..., nc - 1]),
                     ("mass", lambda p, nc: p[..., 0] / p[..., nc - 1])):
        num = den = 0.0
        for ba, bb in zip(a, b):
            for f, pa, pb in zip(case.families, ba, bb):
                xa, xb = fn(pa[2:-2, 2:-2, 2:-2], f.nc), fn(pb[2:-2, 2:-2, 2:-2], f.nc)
                num += float(np.abs(xa - xb).sum()); den += float(np.abs(xb).sum())
        out[name] = num / den
    return out


def jets_capped(prec):
    """The jets case with the time step capped below its CFL value in both forms. The domain starts
    empty (density 1e-20) and the global CFL condition includes empty cells. In the plain form, a
    nearly empty cell beside an entering jet takes a velocity that is FP64 rounding noise over a
    density near 1e-22 (hundreds of m/s), and that cell sets dt from the third step on (2e-7 s
    against 2e-5 s in the FP32 form, whose upwind-split flux keeps those velocities bounded). With
    dt_max below both, both forms take the same steps and the comparison measures the flux and
    source precision alone."""
    c = configs.jets_2d(n=128, steps=100, precision=prec)
    c.numerics.dt_max = 1e-7
    return c


@pytest.mark.parametrize("make", [
    lambda prec: configs.cloud_3d(n=32, steps=20, length=0.0032, precision=prec),
    lambda prec: configs.multiblock_tree(nblocks=6, seed=3, lo=8, hi=16, steps=20, precision=prec),
    jets_capped,
    lambda prec: configs.taylor_green_ig(n=48, steps=20, precision=prec),
], ids=["cloud3d", "multiblock", "jets2d", "taylorgreen"])
def test_fp32_flux_form_within_1e4_l1(gpu, make):
    c32, c64 = make(abi.PREC_FP32FLUX), make(abi.PREC_FP64)
    s32, s64 = Solver(c32, gpu), Solver(c64, gpu)
    steps = c64.numerics.itermax
    o32, o64 = s32.step(steps), s64.step(steps)
    assert o32.status == 0 and o64.status == 0
    assert abs(o32.time - o64.time) <= 1e-3 * o64.time
    if make is jets_capped:
        assert o32.dtglobal == o64.dtglobal == 1e-7
    err = rel_l1(s32.download_all(), s64.download_all(), c64)
    for k, v in err.items():
        assert v <= 1e-4, (k, v)
