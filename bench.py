"""Benchmark of the solve stage on B200: cell-updates/s of ICE's dispersed-phase time step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload multiblock48|cloud192|jets1024|riemann2000]

One "step" is one full time step (every family, every RK stage) of the workload. The default
workload is the 3-D multi-block evaporating case (48 blocks of U[16,160] cells per axis, seed 9,
39.1 M cells, MK + IG + AG families, drag, heat, radiation, evaporation with Langmuir-Knudsen
and blowing, MUSCL van Leer + Jameson sensor, SSP-RK3). The chosen form (FP32 reconstruction,
fluxes and sources; FP64 accumulation, dt and norms) is the headline `value`; the plain FP64 form
runs on the same inputs beside it, and the L1 error of the chosen form against it is reported.

N > 1 (torchrun): every rank advances its own replica of the workload (no exchange); value is
the cell-updates of all ranks over the slowest rank's device time.

--impl reference: the reference's FP64 CPU path, restated by the oracle (the reference's Fortran
cannot be built here: no Fortran compiler, no FiNeR, no ORION), on every host core, on a bounded
sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from ice_b200 import abi, configs  # noqa: E402
from ice_b200.solver import Solver  # noqa: E402

KC_STAGE = 4
KC_NAMES = ["dt", "ghost", "beta", "bound", "stage", "irs", "norm"]


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_workload(name: str, precision: int, steps: int):
    if name == "multiblock48":
        return configs.multiblock_tree(steps=steps, precision=precision)
    if name == "cloud192":
        return configs.cloud_3d(n=192, steps=steps, precision=precision)
    if name == "jets1024":
        return configs.jets_2d(n=1024, steps=steps, precision=precision)
    if name == "riemann2000":
        return configs.riemann_1d(n=2000, steps=steps)
    raise SystemExit(f"unknown workload {name}")


def sample_workload(name: str):
    """A bounded sample of the workload for the CPU legs: the first blocks of the same tree, or the
    same case at a reduced size."""
    if name == "multiblock48":
        return configs.multiblock_tree(nblocks=4, steps=1), "first 4 blocks of the seed-9 tree"
    if name == "cloud192":
        return configs.cloud_3d(n=64, steps=1, length=0.0064), "64^3 cut of the same recipe"
    if name == "jets1024":
        return configs.jets_2d(n=256, steps=1), "256^2 of the same recipe"
    return configs.riemann_1d(n=2000, steps=1), "the whole case"


def algorithmic_bytes(case) -> float:
    """Bytes one launch of the stage kernel must move per cell, FP64 state (SURVEY 8(d) per
    stage): read U_(k-1) and U_0, write U_k (24 nc); face normals, areas and lengths of each
    direction and the volume (8 (5 ndir + 1)); the gas and tau of a coupled run (80)."""
    ndir = case.ndir
    per = []
    for f in case.families:
        b = 24 * f.nc + 8 * (5 * ndir + 1) + (80 if case.numerics.coupled else 0)
        if not case.numerics.time_accurate:
            b += 8
        per.append(b)
    return float(np.mean(per))


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows)}


def rel_l1(a_states, b_states, case):
    """Relative L1 error of the chosen form against the plain form: bulk density, number density
    and particle mass (rho/n), summed over every block and family."""
    out = {}
    for name, fn in (("bulk_density", lambda p, nc: p[..., 0]), ("number_density", lambda p, nc: p[..., nc - 1]),
                     ("particle_mass", lambda p, nc: p[..., 0] / p[..., nc - 1])):
        num = den = 0.0
        for ba, bb in zip(a_states, b_states):
            for f, pa, pb in zip(case.families, ba, bb):
                xa = fn(pa[2:-2, 2:-2, 2:-2], f.nc)
                xb = fn(pb[2:-2, 2:-2, 2:-2], f.nc)
                num += float(np.abs(xa - xb).sum())
                den += float(np.abs(xb).sum())
        out[name] = num / max(den, 1e-300)
    return out


def cpu_sample(name, steps=1, threads=0):
    """The oracle (OpenMP, every host core) on a bounded sample: cell-updates/s."""
    import oracle
    orc = oracle.load()
    n = orc.set_threads(threads)
    case, what = sample_workload(name)
    s = Solver(case, orc)
    t = time.perf_counter()
    out = s.step(steps)
    dt = time.perf_counter() - t
    assert out.status == 0
    return case.ncells * steps / dt, n, f"{what}: {case.ncells} cells, {steps} step(s), {dt:.2f} s"


def run_reference(args, rank, world):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    rates = []
    for _ in range(args.warmup):
        cpu_sample(args.workload, 1, cores)
    t_total = 0.0
    desc = ""
    for _ in range(args.steps):
        r, n, desc = cpu_sample(args.workload, 1, cores)
        rates.append(r)
    v = float(statistics.median(rates))
    line = {"metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": args.workload, "form": "FP64 CPU (oracle restatement, OpenMP)"},
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": n, "kind": "port", "sample": desc},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, dist):
    lib = abi.load_gpu()
    # the chosen form and, beside it, the plain FP64 form on the same inputs
    t0 = time.perf_counter()
    case = make_workload(args.workload, abi.PREC_FP32FLUX if args.precision == "fp32flux" else abi.PREC_FP64,
                         args.warmup + args.steps)
    setup_s = time.perf_counter() - t0
    chosen = Solver(case, lib)
    chosen.step(args.warmup)
    if dist:
        dist.barrier()
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        out = chosen.step(args.steps)
    ms = out.device_ms
    if out.status != 0:
        raise SystemExit(f"step status {out.status}")
    if dist:
        import torch
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    cells = case.ncells
    value = cells * args.steps * world / (ms * 1e-3)

    extra = {}
    if rank == 0:
        states_chosen = chosen.download_all()
        # plain FP64 form, same inputs, same steps
        plain_rate = None
        l1 = None
        if args.precision == "fp32flux" and not args.no_plain:
            case.numerics.precision = abi.PREC_FP64
            P = case.params()
            chosen.close()
            plain = Solver(case, lib)
            plain.step(args.warmup)
            o2 = plain.step(args.steps)
            plain_rate = cells * args.steps / (o2.device_ms * 1e-3)
            l1 = rel_l1(states_chosen, plain.download_all(), case)
            plain.close()
            case.numerics.precision = abi.PREC_FP32FLUX
        else:
            chosen.close()
        # stage-kernel roofline: per-class device time of a profiled pass
        prof = Solver(case, lib)
        prof.step(args.warmup)
        lib.set_profiling(prof.ctx, 1)
        nprof = max(2, min(args.steps, 5))
        prof.step(nprof)
        kt = np.zeros(7)
        nl = C.c_int64()
        lib.kernel_times(prof.ctx, abi.ptr(kt), 7, C.byref(nl))
        launches_per_step = nl.value / nprof
        nfam, nrk = len(case.families), case.params().nrk
        stage_ms = kt[KC_STAGE] / (nprof * nfam * nrk)
        bpc = algorithmic_bytes(case)
        achieved = bpc * cells / (stage_ms * 1e-3) / 1e9
        peak, peak_kind = peaks()
        # e2e through the C ABI with host buffers: upload of the states, K steps, download
        states_host = case.state
        h2d = sum(a.nbytes for per in states_host for a in per)
        t_e = time.perf_counter()
        prof.upload(states_host)
        lib.set_profiling(prof.ctx, 0)
        o3 = prof.step(args.steps)
        back = prof.download_all()
        e2e_s = time.perf_counter() - t_e
        d2h = sum(a.nbytes for per in back for a in per)
        prof.close()
        cpu_v, cpu_n, cpu_desc = cpu_sample(args.workload, 1, os.cpu_count() or 1)
        extra = {
            "e2e": {"value": cells * args.steps / e2e_s, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "kernel": "k_stage", "bytes_per_cell": bpc,
                         "note": f"peak of {peak_kind}; achieved = algorithmic bytes / CUDA-event time of the stage kernel"},
            "cpu_baseline": {"value": cpu_v, "unit": "cell-updates/s", "cores": cpu_n, "kind": "port",
                             "sample": cpu_desc},
            "plain_fp64": {"value": plain_rate, "unit": "cell-updates/s"} if plain_rate else None,
            "chosen_vs_plain": (value / world / plain_rate) if plain_rate else None,
            "l1_error_vs_plain": l1,
            "kernel_ms_per_step": {n: round(float(x) / nprof, 4) for n, x in zip(KC_NAMES, kt)},
            "gpu_launches": int(launches_per_step * args.steps),
            "setup_s": round(setup_s, 1),
        }
        line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 flux / f64 accumulate" if args.precision == "fp32flux" else "f64",
                "data": "synthetic (seeded)",
                "config": {"workload": args.workload, "cells": cells, "families": [f.closure for f in case.families],
                           "form": args.precision, "parallelism": f"replicas x{world}",
                           "l2": "inputs larger than L2 (state of every family in HBM, several GB)"},
                "clocks": clk.summary()}
        line.update(extra)
        print(json.dumps(line), flush=True)
    else:
        chosen.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="multiblock48")
    ap.add_argument("--precision", default="fp32flux", choices=["fp64", "fp32flux"])
    ap.add_argument("--no-plain", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl" if args.impl == "ours" else "gloo", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
