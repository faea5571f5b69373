"""The C ABI library: it loads without a GPU, exports every entry point include/ice_gpu.h
declares, and its host-side pairing of block connections (Pair_Connections) is bit-exact
with the oracle's restatement."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from ice_b200 import abi, build, configs

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def gpu_lib():
    build.build()
    return abi.load_gpu()


def test_exports_every_declared_symbol(gpu_lib):
    header = (ROOT / "include" / "ice_gpu.h").read_text()
    declared = sorted(set(re.findall(r"\b(ice_gpu_[a-z_]+)\s*\(", header)))
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(gpu_lib.lib, name), f"{name} is declared but not exported"
    assert sorted(abi.EXPORTED) == declared


def test_struct_layout_matches_header(tmp_path):
    """The ctypes structures have the sizes and field offsets the C compiler gives the header's."""
    import subprocess
    fields = {"ice_gpu_family": abi.Family, "ice_gpu_params": abi.Params, "ice_gpu_step_out": abi.StepOut}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ice_gpu.h"', "int main(void) {"]
    for cname, py in fields.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in fields.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def _pair(lib, case):
    ng = len(case.families)
    rows = case.bc_rows
    ri = np.zeros((len(rows) * ng, abi.REC_INTS), dtype=np.int32)
    for n, (b, i, j, k, f, code, pay) in enumerate(rows):
        for p in range(ng):
            ri[n * ng + p, :7] = (b, i, j, k, f, code, p + 1)
            if code in (101, 201):
                ri[n * ng + p, 7:12] = pay[:5]
    dims = np.array(case.dims, dtype=np.int32).reshape(-1)
    err = C.create_string_buffer(256)
    rc = lib.pair_connections(len(case.nodes), abi.ptr(dims, C.c_int32), ng, ri.shape[0], abi.ptr(ri, C.c_int32), err, 256)
    return rc, ri, err.value.decode()


@pytest.mark.parametrize("nblocks,seed", [(6, 1), (12, 2), (24, 3)])
def test_pairing_bit_exact_with_oracle(gpu_lib, orc, nblocks, seed):
    case = configs.multiblock_tree(nblocks=nblocks, seed=seed, lo=3, hi=7, families=("MK", "IG"))
    rc1, a, e1 = _pair(gpu_lib, case)
    rc2, b, e2 = _pair(orc, case)
    assert rc1 == 0 and rc2 == 0, (e1, e2)
    assert np.array_equal(a, b)
    conn = a[(a[:, 5] == 101)]
    assert len(conn) > 0
    # every face has one owner and one partner that point at each other
    assert np.all(conn[:, 12] > 0)
    owners = conn[conn[:, 13] == 1]
    assert 2 * len(owners) == len(conn)
    partners = a[owners[:, 12] - 1]
    assert np.all(partners[:, 12] - 1 == np.nonzero((a[:, 5] == 101) & (a[:, 13] == 1))[0])


def test_pairing_refuses_a_dangling_connection(gpu_lib, orc):
    case = configs.multiblock_tree(nblocks=3, seed=5, lo=3, hi=5, families=("IG",))
    rows = list(case.bc_rows)
    n = next(q for q, r in enumerate(rows) if r[5] == 101)
    b, i, j, k, f, code, pay = rows[n]
    rows[n] = (b, i, j, k, f, code, (pay[0], pay[1] + 100, pay[2], pay[3], pay[4]))
    case.bc_rows = rows
    rc1, _, e1 = _pair(gpu_lib, case)
    rc2, _, e2 = _pair(orc, case)
    assert rc1 == abi.EINVAL and rc2 == abi.EINVAL
    assert "points at no connection" in e1


def test_create_refuses_saurel_for_gaussian_closures(gpu_lib):
    case = configs.crossing_jets("IG", n=8, steps=1)
    P = case.params()
    P.fam[0].riemann = abi.RIEMANN["Saurel"]
    dims = np.array(case.dims, dtype=np.int32).reshape(-1)
    ctx = C.c_void_p()
    rc = gpu_lib.create(C.byref(P), 1, abi.ptr(dims, C.c_int32), C.byref(ctx))
    assert rc == abi.EINVAL
    assert "Saurel" in gpu_lib.error(None)


def test_chimera_donors_are_checked(orc):
    """ice_gpu_set_chimera refuses donors given to other records, a chimera record without donors
    for a layer, and a donor outside its block's interior; a step refuses to run before the
    donors are set (through the oracle, which shares the ABI)."""
    from ice_b200.solver import Solver, SolveError
    g = dict(np.load(ROOT / "tests" / "golden" / "chimera_IG.npz"))
    case = configs.doisneau_chimera(g, steps=2)
    chim = case.chimera
    case.chimera = {}
    s = Solver(case, orc)
    with pytest.raises(SolveError, match="no donors"):
        s.step(1)
    case.chimera = chim
    case.build_records(orc)
    n = case.chim_n.copy()
    first = int(np.flatnonzero(n[:, 0])[0])
    other = int(np.flatnonzero(n[:, 0] == 0)[0])

    def call(nchi, donor, weight):
        return orc.set_chimera(s.ctx, nchi.shape[0], abi.ptr(nchi, C.c_int32), abi.ptr(donor, C.c_int32),
                               abi.ptr(weight))

    bad = n.copy(); bad[other] = (1, 1)
    assert call(bad, case.chim_donor, case.chim_weight) == abi.EINVAL
    bad = n.copy(); bad[first, 1] = 0
    assert call(bad, case.chim_donor, case.chim_weight) == abi.EINVAL
    d = case.chim_donor.copy(); d[0, 1] = 0
    assert call(n, d, case.chim_weight) == abi.EINVAL
    assert call(n, case.chim_donor, case.chim_weight) == abi.OK
    assert s.step(2).status == 0
