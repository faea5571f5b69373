"""The block split of the solve stage over ranks (one GPU per rank): whole blocks per rank by the
reference's longest-processing-time assignment (parallel/Mod_MPI.f90:109-183), and the exchange lists
each rank's step needs at every RK stage (parallel/Mod_GhostExchange.f90:737-893):

- kind CELLS: the two source cells of the ghost layers of every connection record (101, 201) whose
  source block another rank steps: (is, js, ks) and (is, js, ks) + guide(fs). The owner of the source
  block sends them after the stage's state exists; they are written into this rank's copy of that
  block, where the ghost fill reads them as it reads any source cell.
- kind BETA: the Jameson weight of the partner cell of every connection face whose owner record is
  on this rank and whose partner record another rank steps (the owner's face flux takes the smaller
  of the two cells' weights).
- kind FLUX: the flux of every connection face whose owner record is on another rank than its
  partner record: the owner computes it once and sends it.
- kind DT (the step's smallest dt over every rank) and kind NORM (the per-block partial sums of the
  residual norm, every block's from the one rank that steps it) are reductions.

Every list is sorted the same way on the sending and the receiving rank, per pair of ranks, so the
buffers need no indices on the wire. A library applies a plan through ice_gpu_set_partition,
ice_gpu_set_halo and ice_gpu_set_exchange_hook; the hook moves the buffers between ranks.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi

CELLS, BETA, FLUX, DT, NORM = 0, 1, 2, 3, 4
GUIDE = {1: (1, 0, 0), 2: (-1, 0, 0), 3: (0, 1, 0), 4: (0, -1, 0), 5: (0, 0, 1), 6: (0, 0, -1)}


def lpt(weights, nbins: int) -> list:
    """Longest-processing-time assignment: items by descending weight (ties keep their order), each to
    the least-loaded bin (the lowest index among equals). Returns the 0-based bin of every item."""
    order = sorted(range(len(weights)), key=lambda b: -weights[b])     # stable: ties keep their order
    load = [0] * nbins
    owner = [0] * len(weights)
    for b in order:
        r = min(range(nbins), key=lambda q: (load[q], q))
        owner[b] = r
        load[r] += weights[b]
    return owner


@dataclass
class Lists:
    """One kind's lists for one family: per peer rank, the entries sent and received, in buffer order.
    An entry is (b, i, j, k), 1-based, for CELLS and BETA; (cf, 0, 0, 0) for FLUX."""
    send: dict = field(default_factory=dict)
    recv: dict = field(default_factory=dict)

    def flat(self, which):
        d = self.send if which == "send" else self.recv
        rows = [e for q in sorted(d) for e in d[q]]
        return np.array(rows, dtype=np.int32).reshape(-1, 4)

    def counts(self, which):
        d = self.send if which == "send" else self.recv
        return [(q, len(d[q])) for q in sorted(d)]


def _add(d, q, e):
    d.setdefault(q, []).append(e)


def halo_plan(case, owner: list, rank: int) -> dict:
    """{family: {CELLS: Lists, BETA: Lists, FLUX: Lists}} of rank `rank`, from the case's records
    (case.rec_int, built) and the block owners."""
    ri = case.rec_int
    nf = len(case.families)
    plan = {}
    for p in range(nf):
        rows = [n for n in range(ri.shape[0]) if ri[n, 6] == p + 1]
        cells, beta, flux = Lists(), Lists(), Lists()
        need = {}            # (receiver, sender) -> set of cells
        for n in rows:
            b, typ, bs, is_, js, ks, fs = ri[n, 0], ri[n, 5], ri[n, 7], ri[n, 8], ri[n, 9], ri[n, 10], ri[n, 11]
            if typ not in (101, 201):
                continue
            rb, rs = owner[b - 1], owner[bs - 1]
            if rb != rs:
                g = GUIDE[int(fs)]
                for cell in ((bs, is_, js, ks), (bs, is_ + g[0], js + g[1], ks + g[2])):
                    need.setdefault((rb, rs), set()).add(tuple(int(x) for x in cell))
            partner = ri[ri[n, 12] - 1]
            rp = owner[partner[0] - 1]
            if ri[n, 13] == 1 and rp != rb:      # an owner record whose partner another rank steps
                pcell = tuple(int(x) for x in partner[1:4])
                if rb == rank:
                    _add(beta.recv, rp, (int(partner[0]),) + pcell)
                    _add(flux.send, rp, (int(ri[n, 14]), 0, 0, 0))
                if rp == rank:
                    _add(beta.send, rb, (int(partner[0]),) + pcell)
                    _add(flux.recv, rb, (int(ri[n, 14]), 0, 0, 0))
        for (rcv, snd), cs in need.items():
            cs = sorted(cs)
            if rcv == rank:
                cells.recv[snd] = cs
            if snd == rank:
                cells.send[rcv] = cs
        for lst in (beta, flux):
            for d in (lst.send, lst.recv):
                for q in d:
                    d[q] = sorted(d[q])
        plan[p] = {CELLS: cells, BETA: beta, FLUX: flux}
    return plan


def apply_plan(lib, ctx, case, owner: list, rank: int, plan: dict):
    """Hands the partition and every family's lists to a library context."""
    owned = np.array([1 if o == rank else 0 for o in owner], dtype=np.int32)
    rc = lib.set_partition(ctx, abi.ptr(owned, C.c_int32))
    if rc != 0:
        raise RuntimeError(f"set_partition: {lib.error(ctx)}")
    for p, kinds in plan.items():
        for kind, lst in kinds.items():
            s, r = lst.flat("send"), lst.flat("recv")
            s = np.ascontiguousarray(s if s.size else np.zeros((1, 4), np.int32))
            r = np.ascontiguousarray(r if r.size else np.zeros((1, 4), np.int32))
            rc = lib.set_halo(ctx, kind, p + 1, len(lst.flat("send")), abi.ptr(s, C.c_int32),
                              len(lst.flat("recv")), abi.ptr(r, C.c_int32))
            if rc != 0:
                raise RuntimeError(f"set_halo: {lib.error(ctx)}")


def attach_hook(lib, ctx, fn):
    """Hands an EXCHANGE_FN to a library context (the caller keeps fn alive as long as the context)."""
    rc = lib.set_exchange_hook(ctx, C.cast(fn, C.c_void_p), None)
    if rc != 0:
        raise RuntimeError(f"set_exchange_hook: {lib.error(ctx)}")


def split_solver(solver, owner: list, rank: int, dist):
    """Makes a Solver of the whole case step only rank `rank`'s blocks, exchanging over dist
    (torch.distributed, already initialised). Returns the hook object, which must outlive the solver."""
    plan = halo_plan(solver.case, owner, rank)
    apply_plan(solver.lib, solver.ctx, solver.case, owner, rank, plan)
    hook = TorchExchange(dist, solver.case, plan)
    attach_hook(solver.lib, solver.ctx, hook.fn)
    return hook


EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int64, C.POINTER(C.c_double),
                          C.c_int64, C.POINTER(C.c_double))


class TorchExchange:
    """The exchange hook over torch.distributed (gloo on the host, or any backend that moves CPU
    tensors): pairwise sends and receives of each kind's buffers in the plan's per-peer order, a min
    all-reduce for DT and a sum all-reduce for NORM. Every rank calls it at the same points of its
    step, so the collectives match."""

    def __init__(self, dist, case, plan: dict):
        import torch
        self.torch, self.dist, self.case, self.plan = torch, dist, case, plan
        self.fn = EXCHANGE_FN(self._call)
        self.calls = {k: 0 for k in (CELLS, BETA, FLUX, DT, NORM)}

    def _width(self, kind, p):
        return 1 if kind == BETA else self.case.families[p].nc

    def _call(self, user, kind, family, nsend, send, nrecv, recv):
        try:
            torch, dist = self.torch, self.dist
            self.calls[kind] += 1
            if kind in (DT, NORM):
                t = torch.from_numpy(np.ctypeslib.as_array(send, shape=(nsend,)).copy())
                dist.all_reduce(t, op=dist.ReduceOp.MIN if kind == DT else dist.ReduceOp.SUM)
                np.ctypeslib.as_array(recv, shape=(nrecv,))[:] = t.numpy()
                return 0
            p = family - 1
            lst = self.plan[p][kind]
            w = self._width(kind, p)
            sbuf = np.ctypeslib.as_array(send, shape=(max(nsend, 1),))[:nsend]
            rbuf = np.ctypeslib.as_array(recv, shape=(max(nrecv, 1),))[:nrecv]
            reqs, outs, off = [], [], 0
            for q, n in lst.counts("send"):
                t = torch.from_numpy(sbuf[off:off + n * w].copy())
                reqs.append(dist.isend(t, q))
                off += n * w
            off = 0
            for q, n in lst.counts("recv"):
                t = torch.empty(n * w, dtype=torch.float64)
                reqs.append(dist.irecv(t, q))
                outs.append((off, n * w, t))
                off += n * w
            for r in reqs:
                r.wait()
            for o, n, t in outs:
                rbuf[o:o + n] = t.numpy()
            return 0
        except Exception:                       # the library turns a non-zero return into an error
            return 1
