"""The reference's logged GH200 figures that bench.py compares against (REFERENCE_LOGS) must be
the ones in the reference's own logs, as extracted into tests/golden/reference_logs.json by
tests/golden/make_reference_log_fixture.py: the solve times and iteration counts of the Q4
doubling-mesh problem at cycle 20 (67,634,433 DoFs, one GH200) and cycle 22 (269,748,225
DoFs, four GH200), and the setup times."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

FIXTURE = os.path.join(ROOT, "tests", "golden", "reference_logs.json")
DOFS = {20: 67_634_433, 22: 269_748_225}
TABLES = {20: ("fp64", "mixed"), 22: ("fp64_4gpu", "mixed_4gpu")}


@pytest.mark.parametrize("cycle", [20, 22])
def test_reference_figures_match_the_logs(cycle):
    logs = json.load(open(FIXTURE))
    ref = bench.REFERENCE_LOGS[cycle]
    t64, t32 = TABLES[cycle]
    row64 = next(r for r in logs["tables"][t64] if r["dofs"] == DOFS[cycle])
    row32 = next(r for r in logs["tables"][t32] if r["dofs"] == DOFS[cycle])
    # the tables print 4 significant digits, the 'Best timings' lines 5
    assert abs(ref["fp64_mg_seconds"] / row64["cg_time_s"] - 1) < 2e-4
    assert abs(ref["fp32_mg_seconds"] / row32["cg_time_s"] - 1) < 2e-4
    assert ref["iterations"] == row64["cg_its"] == row32["cg_its"]
    assert ref["fp64_mg_setup_seconds"] == logs["setup"][t64][str(cycle)]["seconds"]
    assert ref["fp32_mg_setup_seconds"] == logs["setup"][t32][str(cycle)]["seconds"]
    assert ref["gpus"] == (4 if cycle == 22 else 1)
