"""Benchmark of the solve stage on B200: cell-updates/s of ICE's dispersed-phase time step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload multiblock48|multiblock4|cloud192|cloud96|jets1024|taylorgreen192|riemann2000]
                    [--precision fp32flux|fp64] [--no-plain] [--timed-only] [--surrogate]

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
KC_NAMES = ["dt", "ghost", "beta", "bound", "stage", "irs", "norm", "source"]


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_workload(name: str, precision: int, steps: int):
    if name == "multiblock48":
        return configs.multiblock_tree(steps=steps, precision=precision)
    if name == "multiblock4":   # the first 4 blocks of the same tree (3.7 M cells), the profiling case
        return configs.multiblock_tree(nblocks=4, steps=steps, precision=precision)
    if name == "cloud192":
        return configs.cloud_3d(n=192, steps=steps, precision=precision)
    if name == "cloud96":       # the same recipe at 96^3 (0.88 M cells), the profiling case
        return configs.cloud_3d(n=96, steps=steps, length=0.0096, precision=precision)
    if name == "jets1024":
        return configs.jets_2d(n=1024, steps=steps, precision=precision)
    if name == "taylorgreen192":   # built like the reference's published 192^3 IG benchmark
        return configs.taylor_green_ig(n=192, steps=steps, precision=precision)
    if name == "riemann2000":
        return configs.riemann_1d(n=2000, steps=steps)
    raise SystemExit(f"unknown workload {name}")


def sample_workload(name: str):
    """A bounded sample of the workload for the CPU legs: the first blocks of the same tree, or the
    same case at a reduced size."""
    if name == "multiblock48":
        return configs.multiblock_tree(nblocks=4, steps=1), "the same recipe with 4 blocks (seed 9)"
    if name == "cloud192":
        return configs.cloud_3d(n=64, steps=1, length=0.0064), "64^3 of the same recipe"
    if name == "cloud96":
        return configs.cloud_3d(n=48, steps=1, length=0.0048), "48^3 of the same recipe"
    if name == "jets1024":
        return configs.jets_2d(n=256, steps=1), "256^2 of the same recipe"
    if name == "taylorgreen192":
        return configs.taylor_green_ig(n=64, steps=1), "64^3 of the same recipe"
    return configs.riemann_1d(n=2000, steps=1), "the whole case"


def algorithmic_bytes(case, precision: int = abi.PREC_FP64) -> float:
    """Bytes one launch of the stage kernel must move per cell, averaged over the families and the RK
    stages: read U_(k-1) and U_0 and write U_k (24 nc, FP64 state); per direction the face normal and
    area (32) and the cell length (8) in FP64, or their single-precision copies (16 and 4) in the
    FP32-flux form; the volume (8); the boundary map (4); in a coupled run the nine
    frozen-gas values the fused source reads (72; 36 for their single-precision copy in the FP32-flux
    form) and the relaxation time it writes on the last stage (8 / nrk), or, for an evaporating family
    of a 2-D or 3-D run, the source its own kernel wrote (8 nc; 4 nc in single precision in the FP32-flux
    form); the local dt (8) in steady mode; in 1-D runs the sensor weight (8) when the shock detector
    is on (2-D and 3-D runs evaluate it from the staged density)."""
    ndir = case.ndir
    nrk = case.params().nrk
    per = []
    f32 = precision == abi.PREC_FP32FLUX
    geo = 20 if f32 else 40
    word = 4 if f32 else 8
    for f in case.families:
        b = 24 * f.nc + geo * ndir + 8 + 4
        if case.numerics.coupled:
            b += word * f.nc if (ndir >= 2 and f.evap != "none") else 9 * word + 8 / nrk
        if case.numerics.shock_detector and ndir == 1:
            b += 8
        if not case.numerics.time_accurate:
            b += 8
        per.append(b)
    return float(np.mean(per))


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per cell of one stage-kernel launch, from an
# ncu capture of the 4-block case of the 48-block tree in the chosen form (second RK stage of each
# family, 3,714,802 cells). The 48-block case is the same recipe with the same tile shapes, so its
# launches move about the same bytes per cell: traffic per launch = these x its cells.
DRAM_BYTES_PER_CELL = {"MK": 302.2, "IG": 333.0, "AG": 537.2}


def dram_traffic(case, workload: str, precision: int):
    """Measured DRAM bytes of one stage-kernel launch of the workload (mean over its families), where a
    capture of the same recipe and form exists; None otherwise."""
    if not workload.startswith("multiblock") or precision != abi.PREC_FP32FLUX:
        return None
    return float(np.mean([DRAM_BYTES_PER_CELL[f.closure] for f in case.families])) * case.ncells


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


class CpuSample:
    """The oracle (OpenMP, every host core) on a bounded sample of the workload."""

    def __init__(self, name, threads=0):
        import oracle
        self.orc = oracle.load()
        self.cores = self.orc.set_threads(threads)
        self.case, self.what = sample_workload(name)
        self.solver = Solver(self.case, self.orc)

    def step(self):
        t = time.perf_counter()
        out = self.solver.step(1)
        dt = time.perf_counter() - t
        if out.status != 0:
            raise SystemExit(f"oracle step status {out.status}")
        return self.case.ncells / dt, dt

    def describe(self, secs):
        return f"{self.what}: {self.case.ncells} cells, 1 step per sample, {secs:.2f} s"


def accuracy_leg(lib, steps=100):
    """Part of the CPU-baseline leg: the oracle steps the 48-block tree of the same recipe at U[8, 16]
    cells per axis (seed 9) for 100 steps, as config 4 states them, and both device forms step the
    same case; the per-field relative L1 and L-infinity error of each form against the oracle (every
    slot of every family, and the particle mass), with the oracle's time on every host core."""
    import oracle
    from ice_b200.accuracy import field_errors, worst
    orc = oracle.load()
    cores = orc.set_threads(os.cpu_count() or 1)
    make = lambda prec: configs.multiblock_tree(nblocks=48, lo=8, hi=16, steps=steps, precision=prec)
    ref_case = make(abi.PREC_FP64)
    s = Solver(ref_case, orc)
    t = time.perf_counter()
    o = s.step(steps)
    secs = time.perf_counter() - t
    ref = s.download_all()
    s.close()
    out = {"workload": "48-block tree of the same recipe, U[8, 16] cells per axis (seed 9)",
           "cells": ref_case.ncells, "steps": steps, "oracle_s": round(secs, 1), "oracle_cores": cores,
           "oracle_status": int(o.status)}
    for name, prec in (("plain", abi.PREC_FP64), ("chosen", abi.PREC_FP32FLUX)):
        case = make(prec)
        g = Solver(case, lib)
        og = g.step(steps)
        err = field_errors(case, g.download_all(), ref)
        g.close()
        out[name] = {"status": int(og.status), "time_rel_diff": abs(og.time - o.time) / o.time,
                     "worst_l1_rho_n_mass": worst(err, ("rho", "n", "mass"), "l1"),
                     "worst_linf": worst(err, None, "linf"), "fields": err}
    return out


def run_reference(args, rank, world):
    """The reference arm: rank 0 alone times the FP64 CPU restatement; other ranks do nothing."""
    if rank != 0:
        return
    cs = CpuSample(args.workload, os.cpu_count() or 1)
    for _ in range(args.warmup):
        cs.step()
    rates, secs = [], []
    for _ in range(args.steps):
        r, dt = cs.step()
        rates.append(r)
        secs.append(dt)
    v = float(statistics.median(rates))
    line = {"metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * float(statistics.median(secs)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": args.workload, "form": "FP64 CPU restatement of the reference (OpenMP)"},
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": cs.cores, "kind": "port",
                             "sample": cs.describe(float(statistics.median(secs)))},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def pinned_like(arrays):
    """Page-locked host copies of the state arrays (torch's pinned allocator), or plain copies."""
    try:
        import torch
        out = []
        for a in arrays:
            t = torch.empty(a.shape, dtype=torch.float64).pin_memory()
            v = t.numpy()
            v[...] = a
            out.append((t, v))
        return [v for _, v in out], [t for t, _ in out], True
    except Exception:
        return [np.array(a) for a in arrays], [], False


def e2e_run(lib, case, steps):
    """The step through the C ABI with host buffers, as a driver that keeps its state on the host
    calls it: every step, ice_gpu_step_host uploads every block and family from page-locked host
    memory, steps once and downloads the new state into a second set of host arrays; wall time over
    the whole loop."""
    flat = [a for per in case.state for a in per]
    host, keep, pinned = pinned_like(flat)
    outs, keep2, _ = pinned_like(flat)
    nfam = len(case.families)
    states = [host[b * nfam:(b + 1) * nfam] for b in range(len(case.state))]
    results = [outs[b * nfam:(b + 1) * nfam] for b in range(len(case.state))]
    s = Solver(case, lib)
    s.step_host(states, results, 1)                # warm-up: graphs, staging buffer, streams
    h2d = d2h = 0
    t = time.perf_counter()
    for _ in range(steps):
        s.step_host(states, results, 1)
        h2d += sum(a.nbytes for a in host)
        d2h += sum(a.nbytes for a in outs)
    secs = time.perf_counter() - t
    s.close()
    del keep, keep2
    return case.ncells * steps / secs, h2d // steps, d2h // steps, pinned


def allmax(dist, x: float) -> float:
    """The largest x over the ranks (a device tensor over NCCL, a host tensor over gloo)."""
    if not dist:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(dist, cells: int, steps: int, world: int, ms: float) -> float:
    """Cell-updates/s of the whole job: every rank steps its own replica of `cells` cells, and the job
    takes as long as its slowest rank."""
    return cells * steps * world / (allmax(dist, ms) * 1e-3)


def run_surrogate(args, rank, world, dist):
    """The surrogate-evaporation workload (the 48-block, three-family geometry): every evaporating family
    gets a network trained on 4,194,304 pairs (by default) from the plain closure over the envelope of the initial
    state; the steps then run with it, beside the same steps with the plain FP32 closure. value: cell-
    updates/s with the surrogate; the line adds the fraction of cells the network served and each
    family's training report."""
    lib = abi.load_gpu()
    if args.workload == "multiblock48":        # evaporation active in every cell: droplets everywhere
        case = configs.multiblock_tree(steps=args.warmup + args.steps, precision=abi.PREC_FP32FLUX,
                                       evaporation_everywhere=True)
    else:
        case = make_workload(args.workload, abi.PREC_FP32FLUX, args.warmup + args.steps)
    cells = case.ncells
    sur = Solver(case, lib)
    reports = {}
    for p, fam in enumerate(case.families):
        if fam.evap == "none":
            continue
        o = abi.SurrogateOpts(nsamples=args.surrogate_samples, epochs=args.surrogate_epochs, batch=8192, lr=2e-3,
                              jitter=0.05, seed=17 + p, val_frac=0.02)
        rep = abi.SurrogateReport()
        rc = lib.surrogate_train(sur.ctx, p + 1, C.byref(o), C.byref(rep))
        if rc != 0:
            raise SystemExit(f"surrogate_train: {lib.error(sur.ctx)}")
        reports[fam.closure] = {"train_s": round(rep.seconds, 1), "steps": rep.steps, "val_loss": rep.val_loss,
                                "mdot_rel_median": rep.mdot_rel_median, "mdot_rel_p99": rep.mdot_rel_p99,
                                "q_rel_median": rep.q_rel_median, "q_rel_p99": rep.q_rel_p99}
    sur.step(args.warmup)
    c0 = (C.c_int64 * 3)()
    lib.surrogate_stats(sur.ctx, c0)
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        out = sur.step(args.steps)
    c1 = (C.c_int64 * 3)()
    lib.surrogate_stats(sur.ctx, c1)
    ms = allmax(dist, out.device_ms)
    value = whole_job_rate(dist, cells, args.steps, world, out.device_ms)
    st_sur = sur.download_all()
    sur.close()
    plain = Solver(case, lib)
    plain.step(args.warmup)
    o2 = plain.step(args.steps)
    l1 = rel_l1(st_sur, plain.download_all(), case)
    plain.close()
    n_eval, n_env, n_res = (c1[q] - c0[q] for q in range(3))
    if rank != 0:
        return
    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 flux / f64 accumulate, bf16 surrogate",
            "data": "synthetic (seeded)",
            "config": {"workload": args.workload + "+surrogate", "cells": cells,
                       "families": [f.closure for f in case.families], "form": "fp32flux + surrogate evaporation"},
            "clocks": clk.summary(),
            "surrogate": {"cells_evaluated": n_eval, "served_by_network": n_eval - n_env - n_res,
                          "outside_envelope": n_env, "failed_check": n_res,
                          "plain_closure_value": cells * args.steps / (o2.device_ms * 1e-3),
                          "l1_vs_plain_closure": l1, "training": reports}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, dist):
    lib = abi.load_gpu()
    prec = abi.PREC_FP32FLUX if args.precision == "fp32flux" else abi.PREC_FP64
    t0 = time.perf_counter()
    case = make_workload(args.workload, prec, args.warmup + args.steps)
    setup_s = time.perf_counter() - t0
    cells = case.ncells

    # the timed region: K steps of the chosen form, device time on the library's stream
    chosen = Solver(case, lib)
    chosen.step(args.warmup)
    if dist:
        dist.barrier()
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        out = chosen.step(args.steps)
    if out.status != 0:
        raise SystemExit(f"step status {out.status}")
    ms = allmax(dist, out.device_ms)
    value = whole_job_rate(dist, cells, args.steps, world, out.device_ms)
    if args.timed_only:         # the timed region alone (profiler runs)
        chosen.close()
        if rank == 0:
            print(json.dumps({"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                              "config": {"workload": args.workload, "cells": cells, "form": args.precision},
                              "note": "timed region only"}), flush=True)
        return

    extra = {}
    if rank == 0:
        states_chosen = chosen.download_all()
        chosen.close()
        # the plain FP64 form on the same inputs, and the L1 error of the chosen form against it
        plain_rate = l1 = None
        if prec == abi.PREC_FP32FLUX and not args.no_plain:
            case.numerics.precision = abi.PREC_FP64
            plain = Solver(case, lib)
            plain.step(args.warmup)
            o2 = plain.step(args.steps)
            plain_rate = cells * args.steps / (o2.device_ms * 1e-3)
            l1 = rel_l1(states_chosen, plain.download_all(), case)
            plain.close()
            case.numerics.precision = prec
        del states_chosen
        # per-class device time of a profiled pass (CUDA events around every launch)
        prof = Solver(case, lib)
        prof.step(args.warmup)
        lib.set_profiling(prof.ctx, 1)
        nprof = max(2, min(args.steps, 5))
        prof.step(nprof)
        kt = np.zeros(len(KC_NAMES))
        nl = C.c_int64()
        lib.kernel_times(prof.ctx, abi.ptr(kt), len(KC_NAMES), C.byref(nl))
        prof.close()
        launches_per_step = nl.value / nprof
        nfam, nrk = len(case.families), case.params().nrk
        stage_ms = kt[KC_STAGE] / (nprof * nfam * nrk)
        bpc = algorithmic_bytes(case, prec)
        achieved = bpc * cells / (stage_ms * 1e-3) / 1e9
        peak, peak_kind = peaks()
        traffic = dram_traffic(case, args.workload, prec)
        extra = {
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "traffic_unit": "bytes per launch (ncu DRAM read + write)",
                         "algorithmic_bytes_per_launch": bpc * cells,
                         "kernel": "k_stage3", "bytes_per_cell": bpc,
                         "launch_ms": stage_ms,
                         "note": f"peak of {peak_kind}; achieved = algorithmic bytes per launch / mean CUDA-event "
                                 f"duration of the stage kernel's launches"},
            "plain_fp64": {"value": plain_rate, "unit": "cell-updates/s"} if plain_rate else None,
            "chosen_vs_plain": (value / world / plain_rate) if plain_rate else None,
            "l1_error_vs_plain": l1,
            "kernel_ms_per_step": {n: round(float(x) / nprof, 4) for n, x in zip(KC_NAMES, kt)},
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "setup_s": round(setup_s, 1),
        }
    else:
        chosen.close()
    if dist:
        dist.barrier()

    # end to end through the C ABI with host buffers, every rank, slowest rank
    e2e_v, h2d, d2h, pinned = e2e_run(lib, case, args.steps)
    e2e_secs = allmax(dist, cells * args.steps / e2e_v)
    if rank != 0:
        return
    extra["e2e"] = {"value": cells * args.steps * world / e2e_secs, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "host_memory": "pinned" if pinned else "pageable",
                    "form": "every step: ice_gpu_step_host (upload of every block and family, one step, download; "
                            "the copies overlap the other families' stages)"}
    if world == 1:
        if args.workload == "multiblock48" and not args.no_plain:
            extra["accuracy_vs_oracle"] = accuracy_leg(lib)
        cs = CpuSample(args.workload, os.cpu_count() or 1)
        cs.step()
        n, secs = 0, 0.0
        while secs < 10.0 and n < 50:          # about ten seconds of host work
            secs += cs.step()[1]
            n += 1
        extra["cpu_baseline"] = {"value": cs.case.ncells * n / secs, "unit": "cell-updates/s", "cores": cs.cores,
                                 "kind": "port", "sample": f"{cs.what}: {cs.case.ncells} cells, {n} step(s), "
                                                           f"{secs:.1f} s"}
    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 flux / f64 accumulate" if prec == abi.PREC_FP32FLUX else "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "cells": cells, "families": [f.closure for f in case.families],
                       "form": args.precision, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (the state of every family is several GB in HBM)"},
            "clocks": clk.summary()}
    line.update(extra)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="multiblock48")
    ap.add_argument("--precision", default="fp32flux", choices=["fp64", "fp32flux"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 form beside the chosen one")
    ap.add_argument("--timed-only", action="store_true", help="only the timed steps (for profiler runs)")
    ap.add_argument("--surrogate", action="store_true", help="the surrogate-evaporation workload (networks trained first)")
    ap.add_argument("--surrogate-samples", type=int, default=1 << 22, help="training pairs per evaporating family")
    ap.add_argument("--surrogate-epochs", type=int, default=20)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    if args.surrogate:
        run_surrogate(args, rank, world, dist)
    else:
        run_ours(args, rank, world, dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
