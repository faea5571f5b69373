"""The host side of the solve stage: one context of a library that implements the
ABI of include/ice_gpu.h, fed from a Case the way the Fortran driver feeds it
(Wrap_Setup.f90:94-121 for the set-up, Wrap_Solve.f90:26 for each step).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .case import Case


class SolveError(RuntimeError):
    pass


class Solver:
    def __init__(self, case: Case, lib: abi.Backend | None = None, upload: bool = True):
        self.case = case
        self.lib = lib if lib is not None else abi.load_gpu()
        if not case.geoms:
            case.build_geometry()
        if case.rec_int is None:
            case.build_records(self.lib)
        self.freeze_note = case.setup_freeze()
        self.params = case.params()
        dims = np.array(case.dims, dtype=np.int32).reshape(-1)
        ctx = C.c_void_p()
        rc = self.lib.create(C.byref(self.params), len(case.nodes), abi.ptr(dims, C.c_int32), C.byref(ctx))
        if rc != 0:
            raise SolveError(f"create failed ({rc}): {self.lib.error(None)}")
        self.ctx = ctx
        self.last = abi.StepOut()
        for b, g in enumerate(case.geoms):
            self._check(self.lib.set_block(ctx, b + 1, abi.ptr(g.face[0]), abi.ptr(g.face[1]), abi.ptr(g.face[2]),
                                           abi.ptr(g.vol), abi.ptr(g.dl), abi.ptr(g.M)), "set_block")
        self._check(self.lib.set_records(ctx, case.rec_int.shape[0], abi.ptr(case.rec_int, C.c_int32),
                                         abi.ptr(case.rec_real)), "set_records")
        if case.chim_n is not None:
            self._check(self.lib.set_chimera(ctx, case.chim_n.shape[0], abi.ptr(case.chim_n, C.c_int32),
                                             abi.ptr(case.chim_donor, C.c_int32), abi.ptr(case.chim_weight)),
                        "set_chimera")
        for b, gas in enumerate(case.gas):
            self._check(self.lib.set_gas(ctx, b + 1, abi.ptr(gas["prim5"]), abi.ptr(gas["R"]), abi.ptr(gas["gam"]),
                                         abi.ptr(gas["k"]), abi.ptr(gas["mu"])), "set_gas")
        if upload:
            self.upload()

    def _check(self, rc, what):
        if rc != 0:
            raise SolveError(f"{what} failed ({rc}): {self.lib.error(self.ctx)}")

    def upload(self, states=None):
        states = states if states is not None else self.case.state
        for b, per_fam in enumerate(states):
            for p, prim in enumerate(per_fam):
                a = np.ascontiguousarray(prim, dtype=np.float64)
                self._check(self.lib.upload_state(self.ctx, b + 1, p + 1, abi.ptr(a), None), "upload_state")

    def download(self, b: int, p: int) -> np.ndarray:
        ni, nj, nk = self.case.dims[b]
        out = np.empty((nk + 4, nj + 4, ni + 4, self.case.families[p].nc))
        self._check(self.lib.download_state(self.ctx, b + 1, p + 1, abi.ptr(out)), "download_state")
        return out

    def download_all(self):
        return [[self.download(b, p) for p in range(len(self.case.families))] for b in range(len(self.case.nodes))]

    def step(self, nsteps: int = 1, check: bool = True) -> abi.StepOut:
        rc = self.lib.step(self.ctx, nsteps, C.byref(self.last))
        if check and rc != 0:
            raise SolveError(f"step failed ({rc}, status {self.last.status}): {self.lib.error(self.ctx)}")
        return self.last

    def step_host(self, states_in, states_out, nsteps: int = 1, check: bool = True) -> abi.StepOut:
        """ice_gpu_step_host: the state in and out of host arrays, per block and family in the layout
        of upload/download (C-contiguous float64; page-locked for full-speed copies). states_out may
        be states_in."""
        nf = len(self.case.families)
        flat_in = [a for per in states_in for a in per]
        flat_out = [a for per in states_out for a in per]
        assert len(flat_in) == len(flat_out) == len(self.case.nodes) * nf
        for a in flat_in + flat_out:
            assert a.dtype == np.float64 and a.flags.c_contiguous
        P = C.POINTER(C.c_double)
        pin = (P * len(flat_in))(*[abi.ptr(a) for a in flat_in])
        pout = (P * len(flat_out))(*[abi.ptr(a) for a in flat_out])
        rc = self.lib.step_host(self.ctx, nsteps, pin, pout, C.byref(self.last))
        if check and rc != 0:
            raise SolveError(f"step_host failed ({rc}, status {self.last.status}): {self.lib.error(self.ctx)}")
        return self.last

    def set_time(self, time: float, it: int, it_from_call: int = 0):
        self._check(self.lib.set_time(self.ctx, time, it, it_from_call), "set_time")

    def residual_norm(self):
        tot = np.zeros(5)
        fam = np.zeros(5 * len(self.case.families))
        self._check(self.lib.residual_norm(self.ctx, abi.ptr(tot), abi.ptr(fam)), "residual_norm")
        return tot, fam.reshape(-1, 5)

    def update_params(self, params: abi.Params):
        self._check(self.lib.update_params(self.ctx, C.byref(params)), "update_params")
        self.params = params

    def index_maps(self, p: int):
        nb, nr, no = C.c_int32(), C.c_int32(), C.c_int32()
        self._check(self.lib.index_maps(self.ctx, p + 1, C.byref(nb), None, C.byref(nr), None, C.byref(no), None),
                    "index_maps")
        first = np.zeros(nb.value + 1, np.int32)
        recs = np.zeros(max(nr.value, 1), np.int32)
        own = np.zeros(max(no.value, 1), np.int32)
        self._check(self.lib.index_maps(self.ctx, p + 1, C.byref(nb), abi.ptr(first, C.c_int32), C.byref(nr),
                                        abi.ptr(recs, C.c_int32), C.byref(no), abi.ptr(own, C.c_int32)), "index_maps")
        return first, recs[:nr.value], own[:no.value]

    def close(self):
        if self.ctx:
            self.lib.destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
