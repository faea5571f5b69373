"""The evaporation surrogate on the GPU: the FP32 training kernels' gradient against the CPU
oracle (oracle/mlp.py), the BF16 tensor-core inference against the oracle's forward pass, and a run of
the evaporating cloud with the trained network against the plain closure (FP32 and FP64 forms)."""
import ctypes as C

import numpy as np
import pytest

from ice_b200 import abi, configs
from ice_b200.solver import Solver
from oracle import mlp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from ice_b200 import build
    build.build()
    return abi.load_gpu()


def fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def test_training_gradient_matches_oracle(gpu):
    rng = np.random.default_rng(5)
    w = mlp.glorot(2)
    x = rng.normal(size=(300, mlp.IN)).astype(np.float32)
    t = rng.normal(size=(300, mlp.OUT)).astype(np.float32)
    g = np.zeros(mlp.NPARAM, np.float32)
    loss = np.zeros(1, np.float32)
    assert gpu.mlp_grad(fptr(w), fptr(x), fptr(t), 300, fptr(g), fptr(loss)) == 0, gpu.error(None)
    lo, go = mlp.loss_grad(w.astype(np.float64), x, t)
    assert abs(loss[0] - lo) <= 1e-5 * lo
    for l, (ow, ob) in enumerate(mlp.OFFS):
        i, n = mlp.dims(l)
        for a, b in ((ow, ow + i * n), (ob, ob + n)):
            scale = np.abs(go[a:b]).max()
            err = np.abs(g[a:b] - go[a:b]).max()
            assert err <= 1e-4 * scale + 1e-9, (l, a, err, scale)


def test_tensor_core_inference_matches_oracle(gpu, capsys):
    rng = np.random.default_rng(6)
    w = mlp.glorot(3)
    n = 1000          # four CTAs' worth of 256 rows, the last one partial
    x = rng.normal(size=(n, mlp.IN)).astype(np.float32)
    y = np.zeros((n, 2), np.float32)
    assert gpu.mlp_infer(fptr(w), fptr(x), n, fptr(y)) == 0, gpu.error(None)
    yb = mlp.forward_bf16(w, x)
    y64, _ = mlp.forward(w.astype(np.float64), x)
    scale = np.abs(y64).max()
    # against the same roundings: only the order of the FP32 sums, the hardware exponential and
    # reciprocal of SiLU and the BF16 roundings they tip differ
    with capsys.disabled():
        print(f"\ninference against the same roundings: max {np.abs(y - yb).max() / scale:.2e}, "
              f"median {np.median(np.abs(y - yb)) / scale:.2e} of the output scale")
    assert np.median(np.abs(y - yb)) <= 1e-3 * scale, np.median(np.abs(y - yb)) / scale
    assert np.abs(y - yb).max() <= 1e-2 * scale, np.abs(y - yb).max() / scale
    # against the exact network: the BF16 error of four layers
    assert np.abs(y - y64).max() <= 5e-2 * scale, np.abs(y - y64).max() / scale


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


def test_surrogate_source_against_plain_closure(gpu, capsys):
    """A 32^3 evaporating cloud (AG, Langmuir-Knudsen + blowing): the network is trained on the envelope
    of the initial state, then 20 steps run with it, with the FP32 plain closure and with the FP64 form.
    Every cell is accounted for (network, outside the envelope, or failing the closure check, the last
    two running the plain closure); nearly every cell lies inside the envelope; and the run stays within
    the chosen form's 1e-4 relative L1 of the FP64 form in density, number density and particle mass.
    The fraction of cells the network serves is printed: with BF16 inference its rates are accurate to
    about 1e-3, the check's own tolerance, so the check sends many cells back to the plain closure."""
    make = lambda prec: configs.cloud_3d(n=32, steps=20, length=0.0032, precision=prec)
    sur, f32, f64 = Solver(make(abi.PREC_FP32FLUX), gpu), Solver(make(abi.PREC_FP32FLUX), gpu), Solver(make(abi.PREC_FP64), gpu)
    o = abi.SurrogateOpts(nsamples=1 << 19, epochs=40, batch=4096, lr=2e-3, jitter=0.05, seed=11, val_frac=0.05)
    rep = abi.SurrogateReport()
    assert gpu.surrogate_train(sur.ctx, 1, C.byref(o), C.byref(rep)) == 0, gpu.error(sur.ctx)
    for s in (sur, f32, f64):
        s.step(20)
    cnt = (C.c_int64 * 3)()
    assert gpu.surrogate_stats(sur.ctx, cnt) == 0
    cells, env, res = cnt[0], cnt[1], cnt[2]
    e_sur = rel_l1(sur.download_all(), f64.download_all(), sur.case)
    e_f32 = rel_l1(f32.download_all(), f64.download_all(), sur.case)
    with capsys.disabled():
        print(f"\nsurrogate: train loss {rep.train_loss:.3e}, held-out loss {rep.val_loss:.3e}, "
              f"mass rate error median {rep.mdot_rel_median:.2e} p99 {rep.mdot_rel_p99:.2e}, "
              f"heat rate median {rep.q_rel_median:.2e} p99 {rep.q_rel_p99:.2e}, {rep.seconds:.1f} s")
        print(f"cells {cells}: network {cells - env - res} ({(cells - env - res) / cells:.1%}), outside the "
              f"envelope {env}, failing the check {res}; L1 vs FP64: surrogate {e_sur}, FP32 closure {e_f32}")
    assert cells == 3 * 20 * 32 ** 3
    assert env <= 0.01 * cells, (env, cells)
    assert 0 <= env + res <= cells
    assert rep.mdot_rel_median < 1e-2 and rep.q_rel_median < 1e-2
    # what the network gains: the cells it serves skip the iterative closure
    assert cells - env - res >= 0.1 * cells, (cells - env - res, cells)
    for k, v in e_sur.items():
        assert v <= 1e-4, (k, v)
