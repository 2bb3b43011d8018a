"""The algorithmic FLOP count per cell-step that bench.py reports its compute
roofline with is the count the oracle's counting restatement of the WENO-Z
march tallies."""

import re
from pathlib import Path

from oracle import flops


def test_bench_flop_constant_matches_the_counted_march():
    _, _, total = flops.per_cell_step()
    counted = sum(v for k, v in total.items() if k in ("add", "mul", "div", "sqrt"))
    text = (Path(__file__).resolve().parents[1] / "bench.py").read_text()
    declared = int(re.search(r"^FLOPS_PER_CELL_STEP = (\d+)", text, re.M).group(1))
    assert declared == counted


def test_face_dominates_the_count():
    face, cell, _ = flops.per_cell_step()
    fl = lambda d: sum(v for k, v in d.items() if k in ("add", "mul", "div", "sqrt"))
    # 8 five-point reconstructions are most of a face
    assert fl(face) > 8 * 60 and fl(face) > 10 * fl(cell)
