"""Solution output and restart in the reference's Tecplot layout (ice_b200/output.py): the number format,
the header and the restart counters against the text of the reference's own stored solutions
(tests/golden/tecplot_sample.npz, made by tests/golden/make_golden.py), and a restart through a written
file going on as the uninterrupted run does, bit for bit (the reference's RestartExact gate, its
steady res-threshold and transient legs), on the oracle and on the CUDA path."""
from pathlib import Path

import numpy as np
import pytest

from ice_b200 import abi, configs, output
from ice_b200.solver import Solver

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "tecplot_sample.npz")


def _gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return abi.load_gpu()


@pytest.mark.parametrize("closure", ["MK", "IG", "AG"])
def test_number_format_matches_reference_files(closure):
    """Every sampled value line of the reference's solution, read as a double and printed again, gives
    the same 25 characters."""
    for line in GOLD[f"{closure}_values"]:
        assert output.fortran_e(float(line)) == line
    assert output.fortran_e(0.0) == " 0.00000000000000000E+000"


@pytest.mark.parametrize("closure", ["MK", "IG", "AG"])
def test_header_and_counters_match_reference_files(closure):
    """The VARIABLES and ZONE lines of the crossing-jets case after 5000 steady iterations, and the
    counter lines for the counters the reference stored, are the reference's lines."""
    case = configs.crossing_jets(closure, steps=1)
    assert output.header_lines(case, 0, -5000.0) == list(GOLD[f"{closure}_head"])
    aux = list(GOLD[f"{closure}_aux"])
    values = {l.split()[1]: float(l.split('"')[1]) for l in aux}
    assert output.aux_lines(int(values["CYCLE"]), values) == aux


@pytest.mark.parametrize("closure", ["MK", "IG", "AG"])
def test_layout_matches_reference_files(closure):
    """The reference's own crossing-jets fields (tests/golden/crossing_jets_<closure>.npz), written with the
    case's mesh and the stored counters, give the stored file's lines at the sampled positions: every
    cell line to the character (the order of variables and cells), every node line to 1e-15 of the unit
    domain. The reference's mesh file carries y = 0.060000000000000102 at j = 56, where the case's evenly
    spaced mesh has the double nearest 0.06, so those node lines differ in their last digits."""
    from ice_b200.case import empty_state
    case = configs.crossing_jets(closure, steps=1)
    field = np.load(Path(__file__).resolve().parent / "golden" / f"crossing_jets_{closure}.npz")["field"]
    st = empty_state(case.dims[0], case.families[0].nc)
    for v in range(field.shape[0]):
        st[2, 2:-2, 2:-2, v] = field[v]
    aux = list(GOLD[f"{closure}_aux"])
    values = {l.split()[1]: float(l.split('"')[1]) for l in aux}
    text = output.solution_text(case, [[st]], -5000.0, int(values["CYCLE"]), values).split("\n")
    assert text[:2] == list(GOLD[f"{closure}_head"])
    body = text[2:]
    nn = 3 * int(np.prod([d + 1 for d in case.dims[0]]))
    for n, line in zip(GOLD[f"{closure}_index"], GOLD[f"{closure}_values"]):
        if n < nn:
            assert abs(float(body[n]) - float(line)) <= 1e-15, (n, body[n], line)
        else:
            assert body[n] == line, (n, body[n], line)
    assert text[-7:-1] == aux


def _restart_through_file(lib, tmp_path, make, n, total):
    a = Solver(make(), lib)
    oa = a.step(total)
    b = Solver(make(), lib)
    ob = b.step(n)
    path = tmp_path / "part-field.tec"
    output.write_solution(path, b, ob)
    c = Solver(make(), lib, upload=False)
    output.restart(c, output.read_solution(path))
    oc = c.step(total - n)
    assert oa.iter == oc.iter and oa.todo == oc.todo
    for per_a, per_c in zip(a.download_all(), c.download_all()):
        for x, y in zip(per_a, per_c):
            assert np.array_equal(x[2:-2, 2:-2, 2:-2], y[2:-2, 2:-2, 2:-2])
    return oa, oc


def _restart_checks(lib, tmp_path):
    """steady: the stream res-threshold stops at 444, written at 200 and restarted from the file, stops
    at 444 in the same state (the file carries the residual reference). transient: the three-family
    multi-block case, 10 = 5 + 5 steps, with its time. The file's text is the text of the state."""
    oa, oc = _restart_through_file(lib, tmp_path, lambda: configs.stream_tube("scaling"), 200, 20000)
    assert 200 < oa.iter < 20000 and oa.todo == 3
    oa, oc = _restart_through_file(
        lib, tmp_path, lambda: configs.multiblock_tree(nblocks=4, seed=5, lo=4, hi=7, steps=10), 5, 10)
    assert oa.time == oc.time


def _async_checks(lib, tmp_path):
    """write_solution_async downloads before it returns: stepping on while the host thread writes leaves
    the file holding the state of the step it was asked for."""
    s = Solver(configs.multiblock_tree(nblocks=3, seed=2, lo=4, hi=6, steps=20), lib)
    out = s.step(5)
    t5 = out.time                       # the solver's report is overwritten by its next step
    want = s.download_all()
    fut = output.write_solution_async(tmp_path / "a.tec", s, out)
    s.step(5)
    sol = output.read_solution(fut.result())
    got = output.states_from_solution(s.case, sol)
    for per_w, per_g in zip(want, got):
        for x, y in zip(per_w, per_g):
            assert np.array_equal(x[2:-2, 2:-2, 2:-2], y[2:-2, 2:-2, 2:-2])
    assert sol["aux"]["ICE_ITERATION"] == 5.0 and sol["time"] == t5


def _run_checks(lib, tmp_path):
    """The driver's loop: a 12-iteration run with a solution every 5 writes at 5, 10 and 12, the last
    file holding the final state; a steady run ends on res-threshold at 444 with its counters in the
    file."""
    s = Solver(configs.multiblock_tree(nblocks=3, seed=2, lo=4, hi=6, steps=12), lib)
    s.case.numerics.sol_diter = 5
    s.update_params(s.case.params())
    assert output.run(s, str(tmp_path)) == [5, 10, 12]
    sol = output.read_solution(tmp_path / "part-field.tec")
    for per_w, per_g in zip(s.download_all(), output.states_from_solution(s.case, sol)):
        for x, y in zip(per_w, per_g):
            assert np.array_equal(x[2:-2, 2:-2, 2:-2], y[2:-2, 2:-2, 2:-2])
    assert sol["aux"]["ICE_ITERATION"] == 12.0 and sol["aux"]["ICE_OUTPUT_NUMBER"] == 2.0
    s = Solver(configs.stream_tube("scaling"), lib)
    written = output.run(s, str(tmp_path))
    sol = output.read_solution(tmp_path / "part-field.tec")
    ref = np.zeros(1)
    assert lib.get_res_reference(s.ctx, abi.ptr(ref)) == abi.OK
    assert written == [s.last.iter] and 200 < written[0] < 20000
    assert sol["time"] == -float(written[0]) and sol["aux"]["ICE_RES_REFERENCE"] == ref[0]


def test_run_loop_oracle(orc, tmp_path):
    _run_checks(orc, tmp_path)


def test_restart_through_file_oracle(orc, tmp_path):
    _restart_checks(orc, tmp_path)


def test_async_output_oracle(orc, tmp_path):
    _async_checks(orc, tmp_path)


@pytest.mark.gpu
def test_restart_through_file_gpu(tmp_path):
    _restart_checks(_gpu(), tmp_path)


@pytest.mark.gpu
def test_async_output_gpu(tmp_path):
    _async_checks(_gpu(), tmp_path)


@pytest.mark.gpu
def test_run_loop_gpu(tmp_path):
    _run_checks(_gpu(), tmp_path)
