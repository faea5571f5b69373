"""The entry point that allocates nothing, ice_gpu_residual_sq_noalloc, against the residual norm of a
solve context.

It serves drivers that may not allocate device memory themselves: the host application owns every
device allocation through its own allocator (a coupler running inside a gas solver with a fixed
device-memory budget, or a Fortran/OpenACC runtime holding the state arrays), so they cannot create a
solve context, whose set-up allocates. They already hold a block's new and old state on the device and
ask for the residual of the step. The test plays such a caller: the two states live in device arrays
that the test itself owns (allocated with torch, standing in for the host application's allocator),
and two calls in a row must give the context's residual norm for the same states, within the 1e-12
the parity tests use for the norm.

This file is collected last, so that a run stopping at its first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from ice_b200 import abi, configs
from ice_b200.solver import Solver

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def gpu():
    from ice_b200 import build
    build.build()
    return abi.load_gpu()


def _call(lib, dn, do, nc, dims):
    sums = np.zeros(5)
    err = C.create_string_buffer(256)
    rc = lib.residual_sq_noalloc(C.c_void_p(dn), C.c_void_p(do), nc, nc - 1, abi.ptr(dims, C.c_int32),
                                 abi.ptr(sums), None, err, 256)
    return rc, sums, err.value.decode()


def test_noalloc_residual_matches_context_norm(gpu):
    import torch
    # one block, one AG family of the evaporating-cloud recipe: three steps, the norm of the last
    case = configs.cloud_3d(n=24, steps=3, length=0.0024)
    s = Solver(case, gpu)
    s.step(2)
    old = s.download(0, 0)
    s.step(1)
    new = s.download(0, 0)
    total, _ = s.residual_norm()
    s.close()
    nc = case.families[0].nc
    dims = np.array(case.dims[0], dtype=np.int32)
    # the caller's own device arrays, in the driver's layout prim(nc, -1:ni+2, -1:nj+2, -1:nk+2)
    dn = torch.from_numpy(np.ascontiguousarray(new)).cuda()
    do = torch.from_numpy(np.ascontiguousarray(old)).cuda()
    torch.cuda.synchronize()
    for call in range(2):                      # the scratch keeps the last call's contents
        rc, sums, msg = _call(gpu, dn.data_ptr(), do.data_ptr(), nc, dims)
        assert rc == 0, msg
        got = np.sqrt(sums)
        assert np.all(np.abs(got - total) <= TOL * np.maximum(np.abs(total), 1e-300)), (call, got, total)
    assert float(total[0]) > 0.0, "the step changed nothing: the comparison would be empty"


def test_noalloc_refuses_a_block_beyond_its_scratch(gpu):
    # checked on the host before any launch: the arrays are never read
    dims = np.array([1024, 1024, 9], dtype=np.int32)
    rc, _, msg = _call(gpu, 16, 16, 12, dims)
    assert rc == abi.EINVAL and "8388608" in msg
