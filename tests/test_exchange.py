"""Two-way coupling: the step's source of a family, weighted over the RK stages as the update weighs
them, is what the update integrated; on a uniform cloud in a uniform gas every face flux cancels, so
each cell's change of bulk density over a step is dt times the mass rate the gas receives, negated
(the reference's add_stage_source and exchange_rate: Mod_Explicit.f90:257-300, Mod_Exchange.f90:60-78).
Through the oracle, which shares the C ABI."""
import numpy as np
import pytest

from ice_b200 import abi, configs
from ice_b200.solver import Solver


def _uniform_cloud(scheme, steps=3):
    c = configs.cloud_3d(n=6, steps=steps, length=0.0006)
    c.numerics.scheme = scheme
    st = c.state[0][0]
    st[2:-2, 2:-2, 2:-2, :] = st[4, 4, 4, :].copy()
    gas = c.gas[0]
    gas["prim5"][...] = gas["prim5"][0, 0, 0, :].copy()
    for k in ("R", "gam", "k", "mu"):
        gas[k][...] = gas[k].flat[0]
    return c


@pytest.mark.parametrize("scheme", ["euler", "RK2", "RK3"])
def test_step_source_is_what_the_update_integrated(orc, scheme):
    c = _uniform_cloud(scheme)
    s = Solver(c, orc)
    assert orc.set_exchange(s.ctx, 1) == abi.OK
    m0 = s.download(0, 0)[2:-2, 2:-2, 2:-2, 0].copy()
    out = s.step(1)
    assert out.status == 0
    m1 = s.download(0, 0)[2:-2, 2:-2, 2:-2, 0]
    x = np.zeros((6, 6, 6, 5))
    assert orc.exchange_rate(s.ctx, 1, 1, abi.ptr(x)) == abi.OK
    expect = -x[..., 0] * out.dtglobal
    assert np.max(np.abs(expect)) > 0.0
    assert np.max(np.abs((m1 - m0) - expect)) <= 1e-11 * np.max(np.abs(expect))


def test_exchange_needs_a_coupled_run_and_to_be_on(orc):
    c = _uniform_cloud("RK3")
    s = Solver(c, orc)
    x = np.zeros((6, 6, 6, 5))
    assert orc.exchange_rate(s.ctx, 1, 1, abi.ptr(x)) == abi.ENOTREADY
    u = configs.empty_tube(2)                 # no gas
    su = Solver(u, orc)
    assert orc.set_exchange(su.ctx, 1) == abi.EINVAL
