"""ice_gpu_step_host against upload_state + ice_gpu_step + download_state on the same inputs: the
same bits in every interior cell of every block and family, in both precision forms, for one and for
several steps, with the output arrays separate from the input arrays or the same arrays."""
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


def _case(prec):
    return configs.multiblock_tree(nblocks=6, seed=3, lo=8, hi=16, steps=20, precision=prec)


def _separate_calls(gpu, prec, nsteps):
    s = Solver(_case(prec), gpu)
    out = s.step(nsteps)
    states = s.download_all()
    s.close()
    return out, states


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_FP32FLUX], ids=["fp64", "fp32flux"])
@pytest.mark.parametrize("nsteps", [1, 3])
@pytest.mark.parametrize("in_place", [False, True], ids=["separate", "in_place"])
def test_step_host_matches_the_separate_calls(gpu, prec, nsteps, in_place):
    ref_out, ref = _separate_calls(gpu, prec, nsteps)
    case = _case(prec)
    s = Solver(case, gpu, upload=False)
    ins = [[np.ascontiguousarray(a, dtype=np.float64).copy() for a in per] for per in case.state]
    outs = ins if in_place else [[np.empty_like(a) for a in per] for per in ins]
    out = s.step_host(ins, outs, nsteps)
    assert out.status == ref_out.status == 0
    assert out.iter == ref_out.iter == nsteps
    assert out.time == ref_out.time and out.dtglobal == ref_out.dtglobal
    for per_r, per_o in zip(ref, outs):
        for r, o in zip(per_r, per_o):
            assert np.array_equal(r[2:-2, 2:-2, 2:-2], o[2:-2, 2:-2, 2:-2])
    # a second call continues from the new state, as a driver's next step would
    out2 = s.step_host(outs, outs, 1)
    assert out2.status == 0 and out2.iter == nsteps + 1
    s.close()
