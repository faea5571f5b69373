"""ctypes mirror of include/ice_gpu.h and the loader of the CUDA library.

The structures below are field-for-field the C structures of the ABI; the Fortran
driver binds the same layout through iso_c_binding (ice_b200/fortran/ice_gpu.f90).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

MAX_FAMILIES = 4
NCOND_MAX = 12
NEP = 8
REC_INTS = 15
REC_REALS = 8

OK, EINVAL, ECUDA, ESTATE, ENOMEM, ENOTREADY, EEXCH = 0, 1, 2, 3, 4, 5, 6
ST_NAN_STATE, ST_BAD_RECON, ST_TIMEOUT = 1, 2, 4

CLOSURE = {"MK": 1, "IG": 2, "AG": 3}
NBASE = {1: 6, 2: 7, 3: 12}
RIEMANN = {"Saurel": 1, "Rusanov": 2, "HLLE": 3}
LIMITER = {"IORD": 0, "minmod": 1, "vanalbada": 2, "vanleer": 3, "ospre": 4, "umist": 5, "osher": 6,
           "sweby": 7, "mc": 8, "koren": 9, "superbee": 10}
DRAG = {"Newton": 1, "Stokes": 2, "Schlichting": 3, "Schiller-Naumann": 4, "Wen-Yu": 5, "Putnam": 6,
        "Clift-Gauvin": 7, "Morsi-Alexander": 8, "Carlson-Hoglund": 9, "Henderson": 10, "Crowe": 11,
        "Hermsen": 12, "NoDrag": 13}
HEAT = {"Stokes": 1, "JAXA1": 2, "JAXA2": 3, "JAXA3": 4, "JAXA4": 5, "Ranz-Marshall": 6,
        "Kavanau-Drake": 7, "NoHeat": 8}
EVAP = {"none": 0, "d2-law": 1, "CEM": 2, "CEM-B": 3, "ASM": 4, "TC": 5}
PREC_FP64, PREC_FP32FLUX = 0, 1


class Family(C.Structure):
    _fields_ = [("closure", C.c_int32), ("riemann", C.c_int32), ("nfrozen", C.c_int32),
                ("frozen", C.c_int32 * NCOND_MAX),
                ("rho_al", C.c_double), ("cs_al", C.c_double), ("lv_al", C.c_double), ("emiss", C.c_double),
                ("evap", C.c_int32), ("intf", C.c_int32), ("liq", C.c_int32), ("boil", C.c_int32),
                ("ep", C.c_double * NEP)]


class Params(C.Structure):
    _fields_ = [("nfam", C.c_int32), ("ndir", C.c_int32), ("nrk", C.c_int32), ("time_accurate", C.c_int32),
                ("cfl", C.c_double), ("dt_max", C.c_double), ("tau_factor", C.c_double),
                ("cfl_ramp_iter", C.c_int32), ("limiter", C.c_int32), ("shock_detector", C.c_int32),
                ("irs", C.c_int32), ("irs_beta", C.c_double),
                ("coupled", C.c_int32), ("drag", C.c_int32), ("heat", C.c_int32), ("blow", C.c_int32),
                ("precision", C.c_int32), ("itermax", C.c_int32), ("sol_diter", C.c_int32),
                ("shell_diter", C.c_int32), ("res_diter", C.c_int32), ("no_realize", C.c_int32),
                ("time_threshold", C.c_double), ("res_threshold", C.c_double), ("sol_dtime", C.c_double),
                ("fam", Family * MAX_FAMILIES)]


class StepOut(C.Structure):
    _fields_ = [("dtglobal", C.c_double), ("time", C.c_double), ("iter", C.c_int32), ("todo", C.c_int32),
                ("status", C.c_int32), ("have_norm", C.c_int32), ("nfloored", C.c_int64),
                ("residual", C.c_double * 5), ("device_ms", C.c_double), ("nrealized", C.c_int64)]


class SurrogateOpts(C.Structure):
    _fields_ = [("nsamples", C.c_int64), ("epochs", C.c_int32), ("batch", C.c_int32), ("lr", C.c_double),
                ("jitter", C.c_double), ("seed", C.c_uint64), ("val_frac", C.c_double)]


class SurrogateReport(C.Structure):
    _fields_ = [("train_loss", C.c_double), ("val_loss", C.c_double), ("mdot_rel_median", C.c_double),
                ("mdot_rel_p99", C.c_double), ("q_rel_median", C.c_double), ("q_rel_p99", C.c_double),
                ("seconds", C.c_double), ("nsamples", C.c_int64), ("steps", C.c_int64),
                ("env_lo", C.c_double * 7), ("env_hi", C.c_double * 7)]


MLP_NPARAM = 7 * 128 + 128 + 3 * (128 * 128 + 128) + 128 * 2 + 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_fp = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)
_vp = C.c_void_p


def ptr(a: np.ndarray, ctype=C.c_double):
    return a.ctypes.data_as(C.POINTER(ctype))


# name, restype, argtypes (ctx first where the call takes one)
_SIGNATURES = [
    ("create", C.c_int, [C.POINTER(Params), C.c_int32, _ip, C.POINTER(_vp)]),
    ("set_block", C.c_int, [_vp, C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp]),
    ("set_records", C.c_int, [_vp, C.c_int32, _ip, _dp]),
    ("set_chimera", C.c_int, [_vp, C.c_int32, _ip, _ip, _dp]),
    ("set_imports", C.c_int, [_vp, C.c_int32, C.c_int32, _dp]),
    ("set_exchange", C.c_int, [_vp, C.c_int32]),
    ("exchange_rate", C.c_int, [_vp, C.c_int32, C.c_int32, _dp]),
    ("set_gas", C.c_int, [_vp, C.c_int32, _dp, _dp, _dp, _dp, _dp]),
    ("upload_state", C.c_int, [_vp, C.c_int32, C.c_int32, _dp, _u8p]),
    ("download_state", C.c_int, [_vp, C.c_int32, C.c_int32, _dp]),
    ("set_time", C.c_int, [_vp, C.c_double, C.c_int32, C.c_int32]),
    ("set_res_reference", C.c_int, [_vp, C.c_double]),
    ("get_res_reference", C.c_int, [_vp, _dp]),
    ("step", C.c_int, [_vp, C.c_int32, C.POINTER(StepOut)]),
    ("residual_norm", C.c_int, [_vp, _dp, _dp]),
    ("update_params", C.c_int, [_vp, C.POINTER(Params)]),
    ("last_error", C.c_int, [_vp, C.c_char_p, C.c_int32]),
    ("destroy", C.c_int, [_vp]),
    ("pair_connections", C.c_int, [C.c_int32, _ip, C.c_int32, C.c_int32, _ip, C.c_char_p, C.c_int32]),
    ("index_maps", C.c_int, [_vp, C.c_int32, _ip, _ip, _ip, _ip, _ip, _ip]),
    ("set_partition", C.c_int, [_vp, _ip]),
    ("set_halo", C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, _ip, C.c_int32, _ip]),
    ("set_exchange_hook", C.c_int, [_vp, _vp, _vp]),
]
GPU_ONLY = [
    ("step_host", C.c_int, [_vp, C.c_int32, C.POINTER(_dp), C.POINTER(_dp), C.POINTER(StepOut)]),
    ("set_profiling", C.c_int, [_vp, C.c_int32]),
    ("kernel_times", C.c_int, [_vp, _dp, C.c_int32, C.POINTER(C.c_int64)]),
    ("residual_sq_noalloc", C.c_int, [_vp, _vp, C.c_int32, C.c_int32, _ip, _dp, _vp, C.c_char_p, C.c_int32]),
    ("surrogate_train", C.c_int, [_vp, C.c_int32, C.POINTER(SurrogateOpts), C.POINTER(SurrogateReport)]),
    ("surrogate_enable", C.c_int, [_vp, C.c_int32, C.c_int32]),
    ("surrogate_stats", C.c_int, [_vp, C.POINTER(C.c_int64)]),
    ("mlp_grad", C.c_int, [_fp, _fp, _fp, C.c_int32, _fp, _fp]),
    ("mlp_infer", C.c_int, [_fp, _fp, C.c_int32, _fp]),
]

# every symbol include/ice_gpu.h declares
EXPORTED = ["ice_gpu_" + n for n, _, _ in _SIGNATURES + GPU_ONLY]


class Backend:
    """One library implementing the ABI: the CUDA product (prefix ice_gpu_) or a
    restatement with the same entry points under another prefix."""

    def __init__(self, path: str | os.PathLike, prefix: str, extra=()):
        self.path = str(path)
        self.lib = C.CDLL(self.path)
        self.prefix = prefix
        for name, res, args in list(_SIGNATURES) + list(extra):
            fn = getattr(self.lib, prefix + name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
            setattr(self, name, fn)

    def error(self, ctx) -> str:
        buf = C.create_string_buffer(1024)
        self.last_error(ctx, buf, 1024)
        return buf.value.decode(errors="replace")


_PKG = Path(__file__).resolve().parent
GPU_LIB = _PKG / "lib" / "libice_gpu.so"


def load_gpu() -> Backend:
    """The CUDA library. Raises if it has not been built: there is no fallback."""
    if not GPU_LIB.exists():
        raise RuntimeError(f"{GPU_LIB} is missing: build it with `python -m ice_b200.build` "
                           "(the solve stage has no CPU fallback)")
    return Backend(GPU_LIB, "ice_gpu_", extra=GPU_ONLY)
