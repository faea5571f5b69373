"""The tuner of the staged stage kernel's schedule: for each closure it times the kernel on one GPU for
every candidate (kz, zpass, wcap) of ice_b200/csrc/ice_tune.h and writes the fastest into that file,
with the measurements, for the library's next build.

    python -m ice_b200.tune [--blocks 8] [--steps 3] [--out ice_b200/csrc/ice_tune.h] [--dry]

The workload is the 48-block tree's recipe (seed 9, blocks of U[16, 160] cells per axis) cut to its
first --blocks blocks, one family at a time in the chosen form (FP32 fluxes, FP64 accumulation),
so that each closure's kernel is timed on the block shapes it meets. A candidate is applied through
ICE_GPU_TUNE, which the library reads when a context is created; the time is the mean CUDA-event
duration of the stage kernel's launches over --steps profiled steps after one warm-up step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import itertools
import json
import os
import sys
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
sys.path.insert(0, str(PKG.parent))

from ice_b200 import abi, configs  # noqa: E402
from ice_b200.solver import Solver  # noqa: E402

CLOSURES = ("MK", "IG", "AG")
KZ = (8, 16, 24, 32)
ZPASS = (1, 2, 3, 4)
WCAP = {"MK": (16, 32, 64), "IG": (16, 32, 64), "AG": (16, 24, 32)}
KC_STAGE = 4


def time_candidate(lib, case, steps: int) -> float:
    s = Solver(case, lib)
    s.step(1)
    lib.set_profiling(s.ctx, 1)
    s.step(steps)
    kt = np.zeros(8)
    n = C.c_int64()
    lib.kernel_times(s.ctx, abi.ptr(kt), 8, C.byref(n))
    lib.set_profiling(s.ctx, 0)
    s.close()
    return float(kt[KC_STAGE]) / (steps * case.params().nrk)


def header(rows: dict, table: dict, what: str) -> str:
    lines = ["// ice_tune.h -- the staged stage kernel's schedule per closure, as the tuner (ice_b200/tune.py) chose",
             "// it by timing the kernel on one B200. Rewritten by the tuner; the library reads it at build time.",
             "//",
             "//   kz     the most planes one tile's chunk takes (its height is cut into equal chunks of at most kz,",
             "//          fewer when that balances the last wave of CTAs better: choose_kz)",
             "//   zpass  the passes of the CTA per plane that the tile-shape cost adds to the face tasks' passes",
             "//          (the z face and the update): the larger, the more it favours few, full tiles",
             "//   wcap   the widest tile, in owned columns",
             "//",
             "// The environment variable ICE_GPU_TUNE=\"kz,zpass,wcap\" overrides the row of every closure (the",
             "// tuner's sweep uses it).",
             "//",
             f"// Measured: {what}. Stage-kernel launch in ms, the chosen row first:"]
    for cl in CLOSURES:
        ranked = sorted(table[cl].items(), key=lambda kv: kv[1])
        lines.append(f"//   {cl}: " + ", ".join(f"{k} {v:.4f}" for k, v in ranked[:6]) +
                     f"; slowest {ranked[-1][0]} {ranked[-1][1]:.4f}")
    lines += ["#pragma once", "", "namespace ice {", "", "struct TuneRow { int kz, zpass, wcap; };", "",
              "// MK, IG, AG", "constexpr TuneRow kTune[3] = {"]
    for cl in CLOSURES:
        kz, zp, wc = rows[cl]
        lines.append(f"    {{{kz}, {zp}, {wc}}},")
    lines += ["};", "", "}  // namespace ice", ""]
    return "\n".join(lines)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--blocks", type=int, default=8)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--out", default=str(PKG / "csrc" / "ice_tune.h"))
    ap.add_argument("--dry", action="store_true", help="print the table, write nothing")
    args = ap.parse_args()
    lib = abi.load_gpu()
    rows, table = {}, {}
    for cl in CLOSURES:
        case = configs.multiblock_tree(nblocks=args.blocks, steps=10, precision=abi.PREC_FP32FLUX, families=(cl,))
        case.build_geometry()
        case.build_records(lib)
        table[cl] = {}
        for kz, zp, wc in itertools.product(KZ, ZPASS, WCAP[cl]):
            os.environ["ICE_GPU_TUNE"] = f"{kz},{zp},{wc}"
            table[cl][f"({kz},{zp},{wc})"] = time_candidate(lib, case, args.steps)
        os.environ.pop("ICE_GPU_TUNE", None)
        best = min(table[cl].items(), key=lambda kv: kv[1])[0]
        rows[cl] = tuple(int(x) for x in best.strip("()").split(","))
        print(cl, best, f"{table[cl][best]:.4f} ms", flush=True)
    what = (f"the first {args.blocks} blocks of the 48-block tree, {case.ncells} cells, one family at a time, "
            f"FP32-flux form, {args.steps} profiled steps")
    text = header(rows, table, what)
    print(json.dumps({"rows": rows, "table": table}))
    if not args.dry:
        Path(args.out).write_text(text)


if __name__ == "__main__":
    main()
