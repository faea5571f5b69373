"""The stage kernel's tuning table: the tuner (ice_b200/tune.py) writes ice_b200/csrc/ice_tune.h from its
measurements, and the committed table is one it could have written: one row per closure (MK, IG, AG)
inside the limits the library accepts from ICE_GPU_TUNE (1 <= kz <= 32, zpass >= 0, wcap >= 1)."""
import re
from pathlib import Path

from ice_b200 import tune

HEADER = Path(__file__).resolve().parents[1] / "ice_b200" / "csrc" / "ice_tune.h"


def _rows(text):
    body = text[text.index("kTune[3]"):]
    return [tuple(int(x) for x in m) for m in re.findall(r"\{(\d+), (\d+), (\d+)\}", body)]


def test_committed_table_is_well_formed():
    rows = _rows(HEADER.read_text())
    assert len(rows) == 3
    for kz, zp, wc in rows:
        assert 1 <= kz <= 32 and zp >= 0 and wc >= 1


def test_tuner_writes_the_fastest_row():
    table = {cl: {"(16,2,32)": 1.2, "(24,4,64)": 1.0, "(8,1,16)": 1.5} for cl in tune.CLOSURES}
    rows = {cl: (24, 4, 64) for cl in tune.CLOSURES}
    text = tune.header(rows, table, "a test")
    assert _rows(text) == [(24, 4, 64)] * 3
    assert "(24,4,64) 1.0000" in text and "slowest (8,1,16) 1.5000" in text
