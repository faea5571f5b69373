"""TEST INFRASTRUCTURE: the CPU FP64 oracle of ICE's time step (libice_oracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, as the
checker; the product (ice_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

from ice_b200 import abi

HERE = Path(__file__).resolve().parent
LIB = HERE / "libice_oracle.so"


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime
                                        for p in (HERE / "ice_oracle.c", HERE / "ice_oracle_physics.h",
                                                  HERE.parent / "include" / "ice_math.h",
                                                  HERE.parent / "include" / "ice_gpu.h")):
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB


_dp = C.POINTER(C.c_double)
_EXTRA = [
    ("reconstruct", C.c_int, [C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_double, C.c_double, C.c_double,
                              C.c_double, C.c_double, _dp, _dp, C.c_double]),
    ("limiter", C.c_double, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]),
    ("riemann", None, [C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.POINTER(abi.Family)]),
    ("cell_source", C.c_double, [C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_double,
                                 C.POINTER(abi.Family), C.c_int, C.c_int, C.c_int, _dp]),
    ("drag", C.c_double, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]),
    ("heat", C.c_double, [C.c_double, C.c_double, C.c_double, C.c_int]),
    ("evaporation", None, [C.c_double] * 9 + [C.c_int, C.c_int, _dp, _dp, _dp, C.POINTER(C.c_int)]),
    ("blowing", C.c_double, [C.c_double] * 8),
    ("prim2cons", None, [C.c_int, _dp, _dp, C.POINTER(abi.Family)]),
    ("cons2prim", None, [C.c_int, _dp, _dp, C.POINTER(abi.Family)]),
    ("download_aux", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, _dp, _dp, _dp]),
    ("set_threads", C.c_int, [C.c_int]),
    ("math", C.c_double, [C.c_int, C.c_double, C.c_double]),
]


def load() -> abi.Backend:
    return abi.Backend(build(), "orc_", extra=_EXTRA)
