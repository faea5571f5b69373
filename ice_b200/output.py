"""Solution output and restart in the reference's two formats (io/IO_Solution.f90:197-288 writes,
408-445 reads back): the Tecplot ASCII layout of its part-field.tec files, and VTK (sol-format = vtk
raw): a multiblock index part-field.vtm beside one raw-appended XML structured grid per block in vtk/.

The layout, as the reference's stored solutions hold it: a VARIABLES line (x y z, then every family's
primitives named <var>_p<family>), one ZONE per block (I, J, K node counts, DATAPACKING=BLOCK, the
coordinates nodal and the primitives cell-centred, SOLUTIONTIME = the time of a time-accurate run, minus
the iteration count of a steady one), the node coordinates then the cell values with i fastest, one
value per line, and after the last zone the counters a restart reads back, as data set auxiliary data:
CYCLE, ICE_ITERATION, ICE_OUTPUT_NUMBER, ICE_GRID_LEVEL, ICE_LAST_OUTPUT_TIME, ICE_RES_REFERENCE. Every
value is printed with 17 significant digits, so it reads back as the same double.

The VTK layout, as the reference's test readers parse it (test/fast/restart/run.py vtk_time,
test/fast/equiv3d/run.py read_vts): the .vtm lists the block files by file="vtk/<name>_<b>.vts"; each
.vts is a StructuredGrid of WholeExtent "0 ni 0 nj 0 nk" with its arrays in one raw AppendedData section
(each a UInt32 byte count, then little-endian data): field data TIME (the SOLUTIONTIME of the Tecplot
file), CYCLE (Int32) and the five restart counters, the node coordinates as Points, and every family's
primitives <var>_p<family> as Float64 CellData, 8 bytes per cell, i fastest.

write_solution_async overlaps the formatting of a solution with the steps that follow it: the state
is copied off the device first (the download is the only part the next step waits for), and a host
thread formats and writes the file while the device steps on.
"""
from __future__ import annotations

import os
import re
import struct
from concurrent.futures import Future, ThreadPoolExecutor

import numpy as np

from .case import Case, empty_state

NAMES = {"MK": ["rho", "u", "v", "w", "T", "n"],
         "IG": ["rho", "u", "v", "w", "P", "T", "n"],
         "AG": ["rho", "u", "v", "w", "P11", "P12", "P13", "P22", "P23", "P33", "T", "n"]}
COUNTERS = ("ICE_ITERATION", "ICE_OUTPUT_NUMBER", "ICE_GRID_LEVEL", "ICE_LAST_OUTPUT_TIME", "ICE_RES_REFERENCE")


def fortran_e(x: float) -> str:
    """x as the reference's files print it: a blank or a minus, 0. and 17 significant digits, E and a
    signed three-digit exponent (0.10000000000000001E+000 for 0.1)."""
    x = float(x)
    if x == 0.0:
        return (" " if np.copysign(1.0, x) > 0 else "-") + "0.00000000000000000E+000"
    digits = "%.16E" % abs(x)                      # d.ddddddddddddddddE+xx, 17 digits correctly rounded
    mant = digits[0] + digits[2:18]
    exp = int(digits[19:]) + 1
    return ("-" if x < 0 else " ") + "0." + mant + "E" + ("-" if exp < 0 else "+") + "%03d" % abs(exp)


def variable_names(case: Case) -> list:
    return [f"{v}_p{p + 1}" for p, fam in enumerate(case.families) for v in NAMES[fam.closure]]


def header_lines(case: Case, b: int, solution_time: float) -> list:
    """The VARIABLES line (first zone only) and the ZONE line of block b (0-based)."""
    ni, nj, nk = case.dims[b]
    nv = len(variable_names(case))
    zone = (f" ZONE  T = Block{b + 1}, I={ni + 1}, J={nj + 1}, K={nk + 1}, DATAPACKING=BLOCK, "
            f"VARLOCATION=([1-3]=NODAL,[4-{3 + nv}]=CELLCENTERED), SOLUTIONTIME={fortran_e(solution_time).strip()}")
    head = [" VARIABLES = x y z" + "".join("   " + n for n in variable_names(case))] if b == 0 else []
    return head + [zone]


def aux_lines(cycle: int, counters: dict) -> list:
    """The restart counters as data set auxiliary data."""
    out = [f'DATASETAUXDATA CYCLE = "{int(cycle)}"']
    out += [f'DATASETAUXDATA {k} = "{fortran_e(counters[k]).strip()}"' for k in COUNTERS]
    return out


def solution_text(case: Case, states, solution_time: float, cycle: int, counters: dict) -> str:
    """The whole file for the given states (per block, per family, in the layout of upload_state)."""
    lines = []
    for b, nodes in enumerate(case.nodes):
        lines += header_lines(case, b, solution_time)
        for c in range(3):
            lines += [fortran_e(v) for v in nodes[..., c].transpose(2, 1, 0).ravel()]
        for p, fam in enumerate(case.families):
            cells = np.asarray(states[b][p])[2:-2, 2:-2, 2:-2]
            for v in range(fam.nc):
                lines += [fortran_e(x) for x in cells[..., v].ravel()]
    lines += aux_lines(cycle, counters)
    return "\n".join(lines) + "\n"


def _vts_bytes(case: Case, b: int, states, solution_time: float, cycle: int, counters: dict) -> bytes:
    """One block's raw-appended StructuredGrid file."""
    ni, nj, nk = case.dims[b]
    ext = f"0 {ni} 0 {nj} 0 {nk}"
    arrays, heads = [], {"field": [], "points": [], "cell": []}
    off = 0

    def add(section, xml, data: bytes):
        nonlocal off
        heads[section].append(xml.replace("OFFSET", str(off)))
        arrays.append(struct.pack("<I", len(data)) + data)
        off += 4 + len(data)

    add("field", '<DataArray type="Float64" Name="TIME" NumberOfTuples="1" format="appended" offset="OFFSET"/>',
        struct.pack("<d", float(solution_time)))
    add("field", '<DataArray type="Int32" Name="CYCLE" NumberOfTuples="1" format="appended" offset="OFFSET"/>',
        struct.pack("<i", int(cycle)))
    for k in COUNTERS:
        add("field", f'<DataArray type="Float64" Name="{k}" NumberOfTuples="1" format="appended" offset="OFFSET"/>',
            struct.pack("<d", float(counters[k])))
    pts = np.ascontiguousarray(case.nodes[b].transpose(2, 1, 0, 3), dtype="<f8")     # (k, j, i, xyz)
    add("points", '<DataArray type="Float64" Name="Points" NumberOfComponents="3" format="appended" '
                  'offset="OFFSET"/>', pts.tobytes())
    for p, fam in enumerate(case.families):
        cells = np.asarray(states[b][p])[2:-2, 2:-2, 2:-2]
        for v, name in enumerate(NAMES[fam.closure]):
            add("cell", f'<DataArray type="Float64" Name="{name}_p{p + 1}" format="appended" offset="OFFSET"/>',
                np.ascontiguousarray(cells[..., v], dtype="<f8").tobytes())
    head = ['<?xml version="1.0"?>',
            '<VTKFile type="StructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt32">',
            f'  <StructuredGrid WholeExtent="{ext}">',
            "    <FieldData>"] + ["      " + x for x in heads["field"]] + [
            "    </FieldData>",
            f'    <Piece Extent="{ext}">',
            "      <Points>"] + ["        " + x for x in heads["points"]] + [
            "      </Points>",
            "      <CellData>"] + ["        " + x for x in heads["cell"]] + [
            "      </CellData>",
            "    </Piece>",
            "  </StructuredGrid>",
            '  <AppendedData encoding="raw">']
    return ("\n".join(head) + "\n   _").encode("ascii") + b"".join(arrays) + b"\n  </AppendedData>\n</VTKFile>\n"


def write_vtk(vtm_path, case: Case, states, solution_time: float, cycle: int, counters: dict) -> str:
    """The solution in the VTK layout: vtm_path (…/<name>.vtm) and its block files in vtk/ beside it."""
    out_dir, base = os.path.split(os.path.abspath(vtm_path))
    name = base[:-4] if base.endswith(".vtm") else base
    os.makedirs(os.path.join(out_dir, "vtk"), exist_ok=True)
    sets = []
    for b in range(len(case.nodes)):
        rel = f"vtk/{name}_{b + 1}.vts"
        with open(os.path.join(out_dir, rel), "wb") as f:
            f.write(_vts_bytes(case, b, states, solution_time, cycle, counters))
        sets.append(f'    <DataSet index="{b}" name="Block{b + 1}" file="{rel}"/>')
    text = "\n".join(['<?xml version="1.0"?>',
                      '<VTKFile type="vtkMultiBlockDataSet" version="1.0" byte_order="LittleEndian" '
                      'header_type="UInt32">', "  <vtkMultiBlockDataSet>"] + sets +
                     ["  </vtkMultiBlockDataSet>", "</VTKFile>"]) + "\n"
    path = os.path.join(out_dir, name + ".vtm")
    with open(path, "w") as f:
        f.write(text)
    return path


def _vts_arrays(path) -> tuple:
    """{name: (type, bytes)} of every appended array of a .vts, and its (ni, nj, nk)."""
    data = open(path, "rb").read()
    head_end = data.find(b"<AppendedData")
    header = data[:head_end].decode("ascii")
    start = data.find(b"_", head_end) + 1
    e = [int(x) for x in re.search(r'WholeExtent="([^"]+)"', header).group(1).split()]
    out = {}
    for typ, name, off in re.findall(r'<DataArray type="(\w+)" Name="([^"]+)"[^>]*offset="(\d+)"', header):
        o = start + int(off)
        n = struct.unpack("<I", data[o:o + 4])[0]
        out[name] = (typ, data[o + 4:o + 4 + n])
    return out, (e[1] - e[0], e[3] - e[2], e[5] - e[4])


def read_vtk(vtm_path) -> dict:
    """A VTK solution in the dict read_solution gives: per block (I, J, K), node coordinates (I, J, K, 3)
    and cell values (nv, K-1, J-1, I-1) in the order of the file's CellData; TIME; the counters and
    CYCLE as numbers."""
    vtm = open(vtm_path).read()
    root = os.path.dirname(os.path.abspath(vtm_path))
    blocks, time, aux = [], None, {}
    for rel in re.findall(r'file="([^"]+\.vts)"', vtm):
        arr, (ni, nj, nk) = _vts_arrays(os.path.join(root, rel))
        time = struct.unpack("<d", arr["TIME"][1])[0]
        aux["CYCLE"] = float(struct.unpack("<i", arr["CYCLE"][1])[0])
        for k in COUNTERS:
            aux[k] = struct.unpack("<d", arr[k][1])[0]
        pts = np.frombuffer(arr["Points"][1], dtype="<f8").reshape(nk + 1, nj + 1, ni + 1, 3).transpose(2, 1, 0, 3)
        names = [n for n in arr if n not in ("TIME", "CYCLE", "Points") and n not in COUNTERS]
        cells = np.stack([np.frombuffer(arr[n][1], dtype="<f8").reshape(nk, nj, ni) for n in names])
        blocks.append(((ni + 1, nj + 1, nk + 1), np.array(pts), cells))
    return {"blocks": blocks, "time": time, "aux": aux}


def counters_of(solver, out, output_number: int = 0) -> tuple:
    """SOLUTIONTIME, CYCLE and the counters of a solver after a step report `out` (ICE_LAST_OUTPUT_TIME:
    the run's time at this output)."""
    from . import abi
    ref = np.zeros(1)
    rc = solver.lib.get_res_reference(solver.ctx, abi.ptr(ref))
    if rc != 0:
        raise RuntimeError("get_res_reference failed")
    steady = not solver.case.numerics.time_accurate
    time = -float(out.iter) if steady else float(out.time)
    counters = {"ICE_ITERATION": float(out.iter), "ICE_OUTPUT_NUMBER": float(output_number), "ICE_GRID_LEVEL": 1.0,
                "ICE_LAST_OUTPUT_TIME": float(out.time), "ICE_RES_REFERENCE": float(ref[0])}
    return time, int(out.iter), counters


def _write(path, case, states, time, cycle, counters, fmt):
    if fmt == "vtk":
        return write_vtk(path, case, states, time, cycle, counters)
    text = solution_text(case, states, time, cycle, counters)
    with open(path, "w") as f:
        f.write(text)
    return path


def write_solution(path, solver, out, output_number: int = 0, fmt: str = "tecplot"):
    """Download the solver's state and write it with its counters to path (fmt "tecplot": the .tec
    file; "vtk": the .vtm and its block files)."""
    time, cycle, counters = counters_of(solver, out, output_number)
    return _write(path, solver.case, solver.download_all(), time, cycle, counters, fmt)


_POOL = ThreadPoolExecutor(max_workers=1)


def write_solution_async(path, solver, out, output_number: int = 0, fmt: str = "tecplot") -> Future:
    """write_solution with the formatting and the write on a host thread: the state is downloaded now,
    and the solver may step on as soon as this returns. The future's result is the path."""
    time, cycle, counters = counters_of(solver, out, output_number)
    states = solver.download_all()
    case = solver.case
    return _POOL.submit(lambda: _write(path, case, states, time, cycle, counters, fmt))


def read_solution(path) -> dict:
    """The zones of a solution file: per block (I, J, K), node coordinates (I, J, K, 3) and cell values
    (nv, K-1, J-1, I-1); SOLUTIONTIME; the auxiliary data as numbers."""
    text = open(path).read().split("\n")
    zones = [n for n, l in enumerate(text) if l.lstrip().startswith("ZONE")]
    aux = {}
    for l in text:
        m = re.match(r'DATASETAUXDATA\s+(\S+)\s*=\s*"([^"]*)"', l)
        if m:
            aux[m.group(1)] = float(m.group(2))
    nv = len(text[0].split("=", 1)[1].split()) - 3
    blocks, time = [], None
    for z, start in enumerate(zones):
        hdr = text[start]
        g = lambda k: int(re.search(r"\b%s=(\d+)" % k, hdr).group(1))
        I, J, K = g("I"), g("J"), g("K")
        time = float(re.search(r"SOLUTIONTIME=(\S+)", hdr).group(1))
        end = zones[z + 1] if z + 1 < len(zones) else len(text)
        vals = np.array([float(l) for l in text[start + 1:end] if l.strip() and not l.startswith("DATASETAUXDATA")])
        nn, ncl = I * J * K, (I - 1) * (J - 1) * (K - 1)
        nodes = np.stack([vals[c * nn:(c + 1) * nn].reshape(K, J, I).transpose(2, 1, 0) for c in range(3)], axis=-1)
        cells = vals[3 * nn:3 * nn + nv * ncl].reshape(nv, K - 1, J - 1, I - 1)
        blocks.append(((I, J, K), nodes, cells))
    return {"blocks": blocks, "time": time, "aux": aux}


def states_from_solution(case: Case, sol: dict) -> list:
    """The per-block, per-family states of upload_state from a solution: the cell values of the file,
    the ghost cells unset (every step fills both ghost layers before it reads them)."""
    states = []
    for b, (_, _, cells) in enumerate(sol["blocks"]):
        per_fam, v0 = [], 0
        for fam in case.families:
            st = empty_state(case.dims[b], fam.nc)
            st[2:-2, 2:-2, 2:-2, :] = np.moveaxis(cells[v0:v0 + fam.nc], 0, -1)
            per_fam.append(st)
            v0 += fam.nc
        states.append(per_fam)
    return states


def restart(solver, sol: dict):
    """Put a solution into a fresh solver (built with upload=False): the state, the iteration count
    and the residual reference of its counters, and for a time-accurate run its time (read_vtk_tec,
    IO_Solution.f90:408-445)."""
    from . import abi
    solver.upload(states_from_solution(solver.case, sol))
    it = int(sol["aux"]["ICE_ITERATION"])
    time = sol["time"] if solver.case.numerics.time_accurate else sol["aux"]["ICE_LAST_OUTPUT_TIME"]
    solver.set_time(time, it, it)
    solver.last.iter = it                          # the iteration the next output is counted from
    rc = solver.lib.set_res_reference(solver.ctx, sol["aux"]["ICE_RES_REFERENCE"])
    if rc != abi.OK:
        raise RuntimeError("set_res_reference failed")


def read_any(path) -> dict:
    """A solution of either format: a .vtm is read as VTK, anything else as Tecplot ASCII."""
    return read_vtk(path) if str(path).endswith(".vtm") else read_solution(path)


def run(solver, out_dir, chunk: int = 1000, fmt: str = "tecplot") -> list:
    """The driver's loop (Wrap_Solve.f90, ICE_postprocess): step until the step reports the end of the run
    (itermax, time-threshold or res-threshold: todo 3), writing part-field.tec in out_dir at every
    output iteration (sol_diter: todo 2) and at the end, each written on the host thread while the
    steps go on. Steps are taken in calls of up to `chunk`, cut at the next output iteration and at
    itermax (a call ends early only on res-threshold); with a time threshold, one step per call, since
    the step that reaches it is not known ahead. Returns the iterations written, the last at the end
    of the run."""
    nm = solver.case.numerics
    path = os.path.join(out_dir, "part-field.vtm" if fmt == "vtk" else "part-field.tec")
    written, pending, number = [], None, 0
    while True:
        it = solver.last.iter
        n = 1 if nm.time_threshold < 1e30 else min(chunk, max(nm.itermax - it, 1))
        if nm.sol_diter > 0:
            n = min(n, nm.sol_diter - it % nm.sol_diter)
        out = solver.step(n)
        if out.todo in (2, 3):
            if pending is not None:
                pending.result()
            pending = write_solution_async(path, solver, out, number, fmt)
            written.append(int(out.iter))
            number += 1
        if out.todo == 3:
            pending.result()
            return written
