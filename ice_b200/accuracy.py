"""Per-field error of a solution against a reference solution of the same case.

The fields are each family's primitive slots in the reference's order (Assign_Setup.f90:104-117; names
as test/bench/make_case.py:57-62 gives them) plus the particle mass rho / n, over the interior cells
of every block. For a field x with reference x_ref:

    L1   = sum |x - x_ref| / sum |x_ref|
    Linf = max |x - x_ref| / max |x_ref|

(relative to the field's own scale; a field that is zero everywhere in the reference reports the
absolute sum and maximum instead).
"""
from __future__ import annotations

import numpy as np

SLOTS = {
    "MK": ["rho", "u", "v", "w", "T", "n"],
    "IG": ["rho", "u", "v", "w", "P", "T", "n"],
    "AG": ["rho", "u", "v", "w", "P11", "P12", "P13", "P22", "P23", "P33", "T", "n"],
}


def _interior(a):
    return a[2:-2, 2:-2, 2:-2]


def field_errors(case, got, ref) -> dict:
    """got, ref: per block, per family, the downloaded state (Solver.download_all). Returns
    {"<p>:<closure>": {field: {"l1": .., "linf": ..}}} for every family p (1-based)."""
    out = {}
    for p, fam in enumerate(case.families):
        names = SLOTS[fam.closure]
        num = np.zeros(len(names) + 1)
        den = np.zeros(len(names) + 1)
        emax = np.zeros(len(names) + 1)
        rmax = np.zeros(len(names) + 1)
        for bg, br in zip(got, ref):
            a, b = _interior(bg[p]), _interior(br[p])
            fa = [a[..., v] for v in range(fam.nc)] + [a[..., 0] / a[..., fam.nc - 1]]
            fb = [b[..., v] for v in range(fam.nc)] + [b[..., 0] / b[..., fam.nc - 1]]
            for m, (x, y) in enumerate(zip(fa, fb)):
                d = np.abs(x - y)
                num[m] += float(d.sum())
                den[m] += float(np.abs(y).sum())
                emax[m] = max(emax[m], float(d.max()))
                rmax[m] = max(rmax[m], float(np.abs(y).max()))
        fields = {}
        for m, name in enumerate(names + ["mass"]):
            fields[name] = {"l1": num[m] / den[m] if den[m] > 0 else num[m],
                            "linf": emax[m] / rmax[m] if rmax[m] > 0 else emax[m]}
        out[f"{p + 1}:{fam.closure}"] = fields
    return out


def worst(errors: dict, fields=None, norm: str = "l1") -> float:
    """The largest error of the named fields (every field if None) over every family."""
    vals = [e[norm] for fam in errors.values() for name, e in fam.items() if fields is None or name in fields]
    return max(vals) if vals else 0.0
