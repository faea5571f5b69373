"""The block split over ranks (the reference's MPI decomposition, parallel/Mod_MPI.f90:109-183 and
Mod_GhostExchange.f90:737-893), as two gloo ranks on the host: the three-family, multi-block tree with
its connections, drag, heat, radiation, evaporation and the Jameson sensor, split between the ranks by
the longest-processing-time rule, steps to the same bits as one rank stepping every block, with the
same dt and the same residual norm. The exchanges (remote source cells of the ghost layers, partner
Jameson weights, connection fluxes owner -> partner, the dt minimum and the norm's partial sums) go
through the library's hook, here over torch.distributed; the library under test is the oracle, the
FP64 restatement of the reference's step."""
import os
import socket

import numpy as np
import pytest

from ice_b200 import configs, parallel

STEPS = 4


def _case():
    return configs.multiblock_tree(nblocks=6, seed=3, lo=5, hi=10, steps=STEPS)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, steady):
    import datetime
    import torch.distributed as dist
    import oracle
    from ice_b200.solver import Solver
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        orc = oracle.load()
        orc.set_threads(1)
        case = _case()
        case.numerics.time_accurate = not steady
        s = Solver(case, orc)
        owner = parallel.lpt([int(np.prod(d)) for d in case.dims], world)
        hook = parallel.split_solver(s, owner, rank, dist)
        out = s.step(STEPS)
        tot, fam = s.residual_norm()
        states = {f"{b}_{p}": s.download(b, p)[2:-2, 2:-2, 2:-2]
                  for b in range(len(case.nodes)) if owner[b] == rank for p in range(len(case.families))}
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), status=out.status, dt=out.dtglobal, time=out.time,
                 tot=tot, fam=fam, owner=np.array(owner), calls=np.array([hook.calls[k] for k in range(5)]), **states)
        s.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("steady", [False, True], ids=["time_accurate", "steady"])
def test_two_rank_split_steps_to_the_same_bits(orc, tmp_path, steady):
    import torch.multiprocessing as mp
    from ice_b200.solver import Solver
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), steady), nprocs=2, join=True)
    case = _case()
    case.numerics.time_accurate = not steady
    ref = Solver(case, orc)
    out = ref.step(STEPS)
    tot, fam = ref.residual_norm()
    runs = [np.load(tmp_path / f"rank{r}.npz") for r in range(2)]
    owner = list(runs[0]["owner"])
    assert set(owner) == {0, 1}                        # both ranks own blocks
    assert all(r["calls"][parallel.CELLS] > 0 and r["calls"][parallel.FLUX] > 0 for r in runs)
    for r in runs:
        assert int(r["status"]) == 0
        assert float(r["dt"]) == out.dtglobal and float(r["time"]) == out.time
        assert np.array_equal(r["tot"], tot) and np.array_equal(r["fam"], fam)
    for b in range(len(case.nodes)):
        for p in range(len(case.families)):
            got = runs[owner[b]][f"{b}_{p}"]
            assert np.array_equal(got, ref.download(b, p)[2:-2, 2:-2, 2:-2]), (b, p)


def test_lpt_matches_the_reference_rule():
    """lpt_assign (Mod_MPI.f90:146-178): items by descending weight, ties in their order, each to the
    least-loaded bin, the lowest among equals."""
    assert parallel.lpt([5, 9, 9, 1, 4], 2) == [0, 0, 1, 1, 1]     # 9, 9, 5, 4, 1 to bins 0, 1, 0, 1, 1
    assert parallel.lpt([3, 3, 3, 3], 3) == [0, 1, 2, 0]
    w = list(np.random.default_rng(1).integers(1000, 100000, 48))
    owner = parallel.lpt(w, 8)
    loads = [sum(x for x, o in zip(w, owner) if o == r) for r in range(8)]
    assert max(loads) <= sum(w) / 8 + max(w)


class _Loopback:
    """The exchange hook of two ranks that live as two threads of one process, each with its own CUDA
    context on the one GPU: every call posts this rank's send buffer, meets the other rank at a
    barrier and takes the other's buffer (the plan sends everything to the one peer), or reduces both
    for DT (min) and NORM (sum). Each rank's step has drained its stream before it calls the hook, so
    no kernel of one rank waits on the other's; a rank that fails breaks the barrier, which ends the
    other's wait within its timeout."""

    def __init__(self):
        import threading
        self.barrier = threading.Barrier(2, timeout=120)
        self.slot = [None, None]

    def hook(self, rank):
        def call(user, kind, family, nsend, send, nrecv, recv):
            try:
                mine = np.ctypeslib.as_array(send, shape=(max(nsend, 1),))[:nsend].copy()
                self.slot[rank] = mine
                self.barrier.wait()
                other = self.slot[1 - rank]
                out = np.ctypeslib.as_array(recv, shape=(max(nrecv, 1),))[:nrecv]
                if kind == parallel.DT:
                    out[:] = np.minimum(mine, other)
                elif kind == parallel.NORM:
                    out[:] = mine + other if rank == 0 else other + mine
                else:
                    out[:] = other[:nrecv]
                self.barrier.wait()
                return 0
            except Exception:
                self.barrier.abort()
                return 1
        return parallel.EXCHANGE_FN(call)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32flux"])
def test_two_rank_split_on_the_gpu(precision):
    """The CUDA library's split step, two ranks as two contexts on one GPU exchanging through the
    hook: the same bits as one context stepping every block, in both forms."""
    import threading
    import torch
    from ice_b200 import abi
    from ice_b200.solver import Solver
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    gpu = abi.load_gpu()

    def make():
        c = _case()
        c.numerics.precision = precision
        return c
    ref = Solver(make(), gpu)
    out = ref.step(STEPS)
    tot, fam = ref.residual_norm()
    loop = _Loopback()
    owner = parallel.lpt([int(np.prod(d)) for d in ref.case.dims], 2)
    ranks, hooks, results = [], [], [None, None]
    for r in range(2):
        s = Solver(make(), gpu)
        apply = parallel.halo_plan(s.case, owner, r)
        parallel.apply_plan(gpu, s.ctx, s.case, owner, r, apply)
        fn = loop.hook(r)
        parallel.attach_hook(gpu, s.ctx, fn)
        ranks.append(s)
        hooks.append(fn)

    def run(r):
        try:
            o = ranks[r].step(STEPS)
            t, f = ranks[r].residual_norm()
            results[r] = (o.status, o.dtglobal, o.time, t, f)
        except Exception as e:                  # reported below
            results[r] = e
    th = [threading.Thread(target=run, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    for r in range(2):
        assert not isinstance(results[r], Exception), results[r]
        status, dt, time, t, f = results[r]
        assert status == 0 and dt == out.dtglobal and time == out.time
        assert np.array_equal(t, tot) and np.array_equal(f, fam)
    for b in range(len(ref.case.nodes)):
        for p in range(len(ref.case.families)):
            got = ranks[owner[b]].download(b, p)[2:-2, 2:-2, 2:-2]
            assert np.array_equal(got, ref.download(b, p)[2:-2, 2:-2, 2:-2]), (b, p)
