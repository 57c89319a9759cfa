"""Host-side logic of bench.py that needs no GPU: the per-instantiation ratios
against a recorded reference run, and the reference arm's list of cells it
does not run."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_ratios_against_the_recorded_reference_run():
    ref = json.load(open(bench.REFERENCE_CELLS))
    # a run exactly twice as fast as the reference in every warm cell and
    # ten times in every cold one
    mine = {c: {"mops": 2.0 * r["mops"]} for c, r in ref["per_cell"].items()}
    cold = {c: {"mops": 10.0 * r["mops"]} for c, r in ref["cold_per_cell"].items()}
    out = bench.against_reference_cells(mine, cold)
    assert set(out["warm"]) == {c.split(":")[0] for c in ref["per_cell"]}
    for v, r in out["warm"].items():
        assert abs(r["geomean"] - 2.0) < 0.01 and abs(r["min"] - 2.0) < 0.01, (v, r)
    for v, r in out["cold"].items():
        assert abs(r["geomean"] - 10.0) < 0.01, (v, r)
    # cells the reference did not run are left out, not counted as zero
    assert "VAC" not in out["warm"]


def test_reference_arm_skips_the_faulted_instantiation():
    assert "VAC" in bench.REFERENCE_FAULTED
    ref = json.load(open(bench.REFERENCE_CELLS))
    assert not any(c.startswith("VAC:") for c in ref["per_cell"])
