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


def _reference_vtk_time(vtm):
    """The TIME of a VTK solution as the reference's restart test reads it (test/fast/restart/run.py,
    vtk_time): the first block file the .vtm lists, raw appended data, a 4-byte size, then the value."""
    import re
    import struct
    block = re.search(r'file="([^"]+\.vts)"', vtm.read_text()).group(1)
    data = (vtm.parent / block).read_bytes()
    head = data.find(b'<AppendedData')
    m = re.search(rb'Name="TIME"[^>]*offset="(\d+)"', data[:head])
    start = data.find(b'_', head) + 1 + int(m.group(1))
    return struct.unpack('<d', data[start + 4:start + 12])[0]


def _reference_read_vts(path):
    """({name: bytes} of the CellData arrays, (ni, nj, nk)) as the reference's equiv3d test reads a
    raw-appended .vts (test/fast/equiv3d/run.py, read_vts), without decoding."""
    import re
    import struct
    data = Path(path).read_bytes()
    head_end = data.find(b'<AppendedData')
    header = data[:head_end].decode('ascii', 'replace')
    m = re.search(r'header_type="(\w+)"', header)
    hsize = 8 if (m and m.group(1) == 'UInt64') else 4
    hfmt = '<Q' if hsize == 8 else '<I'
    m = re.search(r'WholeExtent="([+-]?\d+) ([+-]?\d+) ([+-]?\d+) ([+-]?\d+) ([+-]?\d+) ([+-]?\d+)"', header)
    e = [int(x) for x in m.groups()]
    dims = (e[1] - e[0], e[3] - e[2], e[5] - e[4])
    start = data.find(b'_', head_end) + 1
    arrays = {}
    cell = header[header.find('<CellData'):header.find('</CellData>')]
    for name, off in re.findall(r'<DataArray[^>]*Name="+([^"]+)"+[^>]*offset="(\d+)"', cell):
        off = start + int(off)
        n = struct.unpack(hfmt, data[off:off + hsize])[0]
        arrays[name] = data[off + hsize:off + hsize + n]
    return arrays, dims


def test_vtk_layout_as_the_reference_reads_it(orc, tmp_path):
    """A VTK solution of the three-family multi-block case, as the reference's own test readers parse it:
    the TIME of the first block file is the solution time; every block file has one CellData array per
    variable of every family, named as the Tecplot file's VARIABLES, each 8 bytes per cell (raw doubles);
    the arrays hold the state (i fastest), and the whole solution reads back to the same bits and
    counters as the Tecplot file of the same state."""
    case = configs.multiblock_tree(nblocks=3, seed=2, lo=4, hi=6, steps=3)
    s = Solver(case, orc)
    out = s.step(3)
    vtm = Path(output.write_solution(tmp_path / "part-field.vtm", s, out, 2, fmt="vtk"))
    tec = Path(output.write_solution(tmp_path / "part-field.tec", s, out, 2))
    assert _reference_vtk_time(vtm) == out.time
    states = s.download_all()
    files = sorted((tmp_path / "vtk").glob("*.vts"))
    assert len(files) == len(case.nodes)
    for b, f in enumerate(sorted(files, key=lambda x: int(x.stem.split("_")[-1]))):
        arrays, dims = _reference_read_vts(f)
        assert dims == tuple(case.dims[b])
        assert list(arrays) == output.variable_names(case)
        v0 = 0
        for p, fam in enumerate(case.families):
            for v in range(fam.nc):
                buf = arrays[output.variable_names(case)[v0 + v]]
                assert len(buf) == 8 * int(np.prod(dims))
                assert np.array_equal(np.frombuffer(buf, dtype="<f8"), states[b][p][2:-2, 2:-2, 2:-2, v].ravel())
            v0 += fam.nc
    a, t = output.read_vtk(vtm), output.read_solution(tec)
    assert a["time"] == t["time"] and a["aux"] == t["aux"]
    for (da, na, ca), (dt, nt, ct) in zip(a["blocks"], t["blocks"]):
        assert da == dt and np.array_equal(na, nt) and np.array_equal(ca, ct)


def _restart_through_file(lib, tmp_path, make, n, total, fmt="tecplot"):
    a = Solver(make(), lib)
    oa = a.step(total)
    b = Solver(make(), lib)
    ob = b.step(n)
    path = tmp_path / ("part-field.vtm" if fmt == "vtk" else "part-field.tec")
    output.write_solution(path, b, ob, fmt=fmt)
    c = Solver(make(), lib, upload=False)
    output.restart(c, output.read_any(path))
    oc = c.step(total - n)
    assert oa.iter == oc.iter and oa.todo == oc.todo
    for per_a, per_c in zip(a.download_all(), c.download_all()):
        for x, y in zip(per_a, per_c):
            assert np.array_equal(x[2:-2, 2:-2, 2:-2], y[2:-2, 2:-2, 2:-2])
    return oa, oc


def _restart_checks(lib, tmp_path):
    """steady: the stream res-threshold stops at 444, written at 200 and restarted from the file, stops
    at 444 in the same state (the file carries the residual reference). transient: the three-family
    multi-block case, 10 = 5 + 5 steps, with its time. In both formats (restart-exact's steady, transient,
    steady-vtk and transient-vtk legs)."""
    for fmt in ("tecplot", "vtk"):
        oa, oc = _restart_through_file(lib, tmp_path, lambda: configs.stream_tube("scaling"), 200, 20000, fmt)
        assert 200 < oa.iter < 20000 and oa.todo == 3
        oa, oc = _restart_through_file(
            lib, tmp_path, lambda: configs.multiblock_tree(nblocks=4, seed=5, lo=4, hi=7, steps=10), 5, 10, fmt)
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
