"""The reference's invariant cases, on the oracle and on the CUDA path, with the gates of their verify.py:
test/NoExchange/MK (an uncoupled cloud keeps its state bit for bit), test/Reflect/AG (x-momentum
conserved along a symmetry plane), test/Thermal/{IG,AG} (the temperature of an expanding blob stays
uniform), test/Axis/{MK,IG,AG} (a one-degree wedge about x: a stationary MK stream keeps its axis
row, IG and AG clouds at rest stay at rest), and test/fast/mirror-modes (the components odd across
mirror faces one cell apart are set to zero at set-up and not integrated)."""
import numpy as np
import pytest

from ice_b200 import abi, configs
from ice_b200.case import SetupError
from ice_b200.solver import Solver


def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return abi.load_gpu()


def _run(case, lib, t_end=None):
    s = Solver(case, lib)
    if t_end is None:
        out = s.step(case.numerics.itermax)
    else:
        out = s.step(1)
        while out.time < t_end * (1.0 - 1e-12):
            assert out.iter < 100000
            out = s.step(1)
    assert out.status == 0
    return out, s.download(0, 0)[2:-2, 2:-2, 2:-2]


def _noexchange(lib, precision=0):
    """NoDrag, NoHeat, no emissivity: density, velocity and temperature stay at their initial values
    bit for bit although the gas moves at 10 m/s and is 100 K hotter (NoExchange/MK/verify.py)."""
    case = configs.noexchange_slab(precision)
    ic = case.state[0][0][2:-2, 2:-2, 2:-2].copy()
    out, st = _run(case, lib)
    assert out.iter == 20
    assert np.array_equal(st[..., :5], ic[..., :5])


def _reflect(lib):
    """The x-momentum sum(rho u V) changes by less than 1e-9 of itself by t = 0.1 (Reflect/AG/verify.py)."""
    case = configs.reflect_blob()
    ic = case.state[0][0][2, 2:-2, 2:-2].copy()
    _, st = _run(case, lib, 0.1)
    v = st[0]
    assert np.isfinite(v).all()
    m0, m1 = float((ic[..., 0] * ic[..., 1]).sum()), float((v[..., 0] * v[..., 1]).sum())
    assert abs(m1 - m0) / m0 < 1e-9


def _thermal(lib, closure):
    """max|T - 1| below 1e-9 over the cells with rho > 1e-3 at t = 0.1, after the blob has expanded to
    max|u| >= 0.1 (Thermal/{IG,AG}/verify.py)."""
    _, st = _run(configs.thermal_blob(closure), lib, 0.1)
    v = st[0]
    assert np.isfinite(v).all()
    live = v[..., 0] > 1e-3
    assert float(np.sqrt((v[..., 1:4] ** 2).sum(-1)).max()) >= 0.1
    assert float(np.abs(v[..., -2][live] - 1.0).max()) < 1e-9


def _axis(lib, closure):
    """MK: after 200 local steps the axis row keeps its initial density to 1e-9 (Axis/MK/verify.py).
    IG, AG: after 500, max(|u|,|v|,|w|)/c, max|rho - 1| and max|Pii - 1| below 1e-10
    (Axis/{IG,AG}/verify.py)."""
    case = configs.axis_wedge(closure)
    ic = case.state[0][0][2, 2:-2, 2:-2].copy()
    out, st = _run(case, lib)
    v = st[0]
    assert out.iter == case.numerics.itermax
    assert np.isfinite(v).all()
    if closure == "MK":
        assert float(np.abs(v[0, :, 0] - ic[0, :, 0]).max()) < 1e-9
        return
    diag = [4] if closure == "IG" else [4, 7, 9]
    c = np.sqrt(3.0 * v[..., 4] / v[..., 0]) if closure == "IG" else np.sqrt(sum(v[..., q] for q in diag) / v[..., 0])
    assert float((np.abs(v[..., 1:4]).max(-1) / c).max()) < 1e-10
    assert float(np.abs(v[..., 0] - 1.0).max()) < 1e-10
    assert max(float(np.abs(v[..., q] - 1.0).max()) for q in diag) < 1e-10


def _mirror_modes(lib):
    """slab (IG, AG): a 2-D layer 1e-5 m thick between wall k faces under cells of 2.5 mm, its odd
    components seeded at 1e-8: after 200 steps w (AG also P13, P23) is zero in every cell, the cloud at
    rest (|u|, |v| below 1e-10), and the set-up's warning names w. tube (IG): a 1-D tube between wall j
    and k faces: v and w zero. A wedge whose k faces are walls instead of 200: the set-up stops and says
    why (mirror-modes/run.py)."""
    for closure, odd in (("IG", [3]), ("AG", [3, 6, 8])):
        s = Solver(configs.mirror_layer("slab", closure), lib)
        assert "2-D plane mesh with mirror k faces: w" in s.freeze_note
        out = s.step(200)
        assert out.status == 0
        v = s.download(0, 0)[2:-2, 2:-2, 2:-2]
        assert all(float(np.abs(v[..., q]).max()) == 0.0 for q in odd)
        assert float(np.abs(v[..., 1:3]).max()) < 1e-10
    s = Solver(configs.mirror_layer("tube", "IG"), lib)
    assert "1-D mesh with mirror j and k faces: v and w" in s.freeze_note
    assert s.step(200).status == 0
    v = s.download(0, 0)[2:-2, 2:-2, 2:-2]
    assert float(np.abs(v[..., 2:4]).max()) == 0.0
    with pytest.raises(SetupError, match="the k faces of an axisymmetric wedge must carry 200"):
        Solver(configs.mirror_layer("wedge", "IG", side_code=300), lib)


def test_mirror_modes_oracle(orc):
    _mirror_modes(orc)


@pytest.mark.gpu
def test_mirror_modes_gpu():
    _mirror_modes(_gpu())


def test_noexchange_oracle(orc):
    _noexchange(orc)


def test_reflect_oracle(orc):
    _reflect(orc)


@pytest.mark.parametrize("closure", ["IG", "AG"])
def test_thermal_oracle(orc, closure):
    _thermal(orc, closure)


@pytest.mark.parametrize("closure", ["MK", "IG", "AG"])
def test_axis_oracle(orc, closure):
    _axis(orc, closure)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_FP32FLUX])
def test_noexchange_gpu(precision):
    _noexchange(_gpu(), precision)


@pytest.mark.gpu
def test_reflect_gpu():
    _reflect(_gpu())


@pytest.mark.gpu
@pytest.mark.parametrize("closure", ["IG", "AG"])
def test_thermal_gpu(closure):
    _thermal(_gpu(), closure)


@pytest.mark.gpu
@pytest.mark.parametrize("closure", ["MK", "IG", "AG"])
def test_axis_gpu(closure):
    _axis(_gpu(), closure)
