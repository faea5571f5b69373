"""Writes the golden fixtures of tests/golden/ from the reference's own test data.

    python tests/golden/make_golden.py /path/to/reference

crossing_jets_{MK,IG,AG}.npz: the fields the reference's own binary wrote after 5000
iterations of its crossing-jets validation cases (test/Doisneau/<closure>/reference/
part-field.tec), every cell-centred variable as float64 in (j, i) order, plus the
boundary table of the case (test/Doisneau/<closure>/INPUT/part-bc.txt) reduced to one
row per record: b i j k f code [alpha] -- so that the test can check the case it builds
against the reference's inputs before comparing fields.

The reference is read here, in this container; the fixtures travel, the reference does not.
"""
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def read_field(path):
    text = Path(path).read_text().split("\n")
    zi = next(i for i, l in enumerate(text) if "ZONE" in l)
    g = lambda k: int(re.search(r"\b%s\s*=\s*(\d+)" % k, text[zi]).group(1))
    I, J, K = g("I"), g("J"), g("K")
    vals = np.array([float(t) for l in text[zi + 1:] if not l.lstrip().startswith("DATASETAUXDATA")
                     for t in l.split()])
    Nn, Nc = I * J * K, (I - 1) * (J - 1) * max(K - 1, 1)
    nv = (len(vals) - 3 * Nn) // Nc
    cells = vals[3 * Nn:3 * Nn + nv * Nc].reshape(nv, max(K - 1, 1), J - 1, I - 1)
    return cells[:, 0]                         # (nv, j, i) of the single k layer


def read_bc(path):
    rows = []
    lines = Path(path).read_text().split("\n")
    q = 0
    while q < len(lines):
        t = lines[q].split()
        q += 1
        if len(t) != 6:
            continue
        b, i, j, k, f, code = map(int, t)
        alpha = 0.0
        if 401 <= code <= 403:
            alpha = float(lines[q].split()[2])
            q += 1
        rows.append((b, i, j, k, f, code, alpha))
    return np.array(rows)


def main(ref):
    ref = Path(ref)
    for cl in ("MK", "IG", "AG"):
        case = ref / "test" / "Doisneau" / cl
        field = read_field(case / "reference" / "part-field.tec")
        bc = read_bc(case / "INPUT" / "part-bc.txt")
        np.savez_compressed(HERE / f"crossing_jets_{cl}.npz", field=field, bc=bc)
        print(cl, field.shape, bc.shape)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
