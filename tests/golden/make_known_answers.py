"""Extract the reference's published known answers for the pressure solve into
`known_answers.json`.  Run once in a container that has the reference source
tree; the JSON is committed so tests never read the reference at run time.

Sources (ronaldremmerswaal/TwoPhaseAMR.jl):
  docs/src/poisson.md:253-257              PCG iterations and L2/Linf errors table
  test/operators/poisson.jl:422-611        root-block hierarchy sizes and stopping
  test/operators/poisson.jl:300-317        Jacobi weight policies
"""
import json
import pathlib
import re
import sys

ROOT = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
doc = (ROOT / "docs/src/poisson.md").read_text().splitlines()
rows = []
for line in doc:
    m = re.match(r"\|\s*(\d+)×(\d+)\s*\|\s*([\d,]+)\s*\|\s*(\d+)\s*\|\s*([\d.e-]+)\s*\|\s*([\d.e-]+)\s*\|", line)
    if m:
        rows.append({"block": int(m.group(1)), "cells": int(m.group(3).replace(",", "")),
                     "pcg_iterations": int(m.group(4)), "l2": float(m.group(5)), "linf": float(m.group(6))})
assert len(rows) == 3, rows
test = (ROOT / "test/operators/poisson.jl").read_text()
assert "expected_bases = [(16, 16), (8, 8), (4, 4)]" in test
assert "expected_sizes = [256, 64, 16]" in test
out = {
    "manufactured_periodic_two_level": {
        "source": "docs/src/poisson.md:253-257; test/operators/poisson.jl:728-831",
        "mesh": "BlockTreeMesh(block_size=(b,b), max_level=2, refine: level 0, or level 1 block (0,0))",
        "rhs": "8 pi^2 sin(2 pi x) cos(2 pi y) at cell centres; exact p = sin(2 pi x) cos(2 pi y)",
        "solver": "EllipticSolver(PoissonOperator(mesh); coarse_size=8), rtol=1e-10, max_cycles=60",
        "rows": rows,
    },
    "root_block_hierarchy": {
        "source": "test/operators/poisson.jl:422-531",
        "base_mesh": [16, 16], "block_size": [4, 4], "coarse_size": 16,
        "expected_bases": [[16, 16], [8, 8], [4, 4]], "expected_sizes": [256, 64, 16],
        "layout_cases": [[[6, 4], [[6, 4], [3, 2]]], [[4, 6], [[4, 6], [2, 3]]], [[3, 4], [[3, 4]]],
                         [[4, 3], [[4, 3]]], [[1, 4], [[1, 4]]], [[4, 1], [[4, 1]]], [[1, 1], [[1, 1]]]],
        "stopping_cases": [[64, 32, [256, 64]], [16, 2, [256, 64]], [16, 1, [256]], [256, 32, [256]]],
        "mixed_pruning": {"base_mesh": [8, 8], "block_size": [4, 4], "max_level": 1,
                          "refine": "level 0 block (0,0)", "coarse_size": 16, "sizes": [112, 64, 16]},
    },
    "periodic_floor": {
        "source": "test/operators/poisson.jl:576-611",
        "cases": [[[8, 8], [True, True], [[8, 8], [4, 4]]], [[4, 4], [False, False], [[4, 4], [2, 2]]],
                  [[8, 4], [True, False], [[8, 4], [4, 2]]], [[4, 8], [False, True], [[4, 8], [2, 4]]]],
        "block_size": [2, 2], "coarse_size": 1,
    },
    "jacobi_weight": {
        "source": "test/operators/poisson.jl:300-317",
        "skip_case": {"diagonal": [2.0, 0.0, -3.0], "row_sums": [1.0, 0.0, 0.0],
                      "inverse": [0.5, 0.0, -3.0], "weight": 4.0 / 1.5},
        "clamped": [[[2.0], [1.0], 1.0], [[2.0], [0.0], 1.0]],
    },
}
(pathlib.Path(__file__).parent / "known_answers.json").write_text(json.dumps(out, indent=1))
print("wrote", len(rows), "table rows")
