"""Extract the reference's logged solver/vmult results into tests/golden/reference_logs.json.

Run once where the reference checkout is available, naming its root:

    REFERENCE_ROOT=<path to the reference checkout> python tests/golden/make_reference_log_fixture.py
    python tests/golden/make_reference_log_fixture.py <path to the reference checkout>

The JSON it writes is committed and is what the tests read.  Each row keeps the file and
line of the log it came from.
"""
import json
import os
import re
import sys

ROOT = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT")
if __name__ == "__main__" and not ROOT:
    sys.exit("name the reference checkout: REFERENCE_ROOT=<path> or the first argument")
LOGS = {
    "fp64": "tests/poisson_cube_bk3_fp64/results/single-gpu-batched.out",
    "mixed": "tests/poisson_cube_bk3/results/signle-gpu-batched-mixed-precision.out",
    # one node, four GPUs over MPI
    "fp64_4gpu": "tests/poisson_cube_bk3_fp64/results/1-node-batched.out",
    "mixed_4gpu": "tests/poisson_cube_bk3/results/1-node-batched-mixed-precision.out",
}


def parse(rel):
    rows = []
    with open(os.path.join(ROOT, rel)) as f:
        lines = f.readlines()
    start = None
    for i, line in enumerate(lines):
        if re.match(r"^\s*cells\s+dofs\s+mv_outer\s+mv_inner\s+cg_time\s+cg_its\s+cg_reduction", line):
            start = i
    if start is None:
        raise SystemExit("table not found in " + rel)
    for j in range(start + 1, len(lines)):
        parts = lines[j].split()
        if len(parts) != 7:
            break
        cells, dofs, mv_o, mv_i, cg_t, its, red = parts
        rows.append({"cells": int(cells), "dofs": int(dofs), "mv_outer_s": float(mv_o),
                     "mv_inner_s": float(mv_i), "cg_time_s": float(cg_t), "cg_its": int(its),
                     "cg_reduction": float(red), "source": f"{rel}:{j + 1}"})
    return rows


def parse_setup(rel):
    """{cycle: {"seconds": total setup time, "source": file:line}} (the first 'Total setup
    time' after each 'Cycle N' line)."""
    out, cycle = {}, None
    with open(os.path.join(ROOT, rel)) as f:
        for j, line in enumerate(f):
            m = re.match(r"^Cycle (\d+)", line)
            if m:
                cycle = int(m.group(1))
                continue
            m = re.search(r"Total setup time: (\S+)", line)
            if m and cycle is not None and str(cycle) not in out:
                out[str(cycle)] = {"seconds": float(m.group(1)), "source": f"{rel}:{j + 1}"}
    return out


def main():
    out = {
        "what": "Q4 ph-multigrid CG on the doubling mesh, f=1, Chebyshev degree 5, range 15, "
                "10 eigenvalue iterations, ReductionControl(100,1e-16,1e-9); logged by the "
                "reference (1 GPU; the *_4gpu tables: one node, 4 GPUs over MPI).",
        "tables": {k: parse(v) for k, v in LOGS.items()},
        "setup": {k: parse_setup(v) for k, v in LOGS.items()},
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_logs.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst, {k: len(v) for k, v in out["tables"].items()})


if __name__ == "__main__":
    sys.exit(main())
