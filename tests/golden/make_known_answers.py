"""Extract the reference's published known answers for the pressure solve into
`known_answers.json`.  Run once, with the path of a TwoPhaseAMR.jl source tree
as the only argument (`python make_known_answers.py <reference checkout>`); the
JSON is committed so tests never read the reference at run time.

Sources (ronaldremmerswaal/TwoPhaseAMR.jl):
  docs/src/poisson.md:253-257              PCG iterations and L2/Linf errors table
  test/operators/poisson.jl:422-611        root-block hierarchy sizes and stopping
  test/operators/poisson.jl:300-317        Jacobi weight policies
  docs/techref/figures/generated/checks.tex  the `chkSolv*` macros that
                                           docs/techref/figures/solvers.jl writes
                                           from the reference's own solves
                                           (iteration counts, convergence factors,
                                           level counts, V-cycle spectra)
"""
import json
import pathlib
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_known_answers.py <TwoPhaseAMR.jl source tree>")
ROOT = pathlib.Path(sys.argv[1])
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
# Chapter 11 of the technical reference: values generated by running the
# reference (solvers.jl asserts them against the chapter's statements).
checks = (ROOT / "docs/techref/figures/generated/checks.tex").read_text()
macros = dict(re.findall(r"\\newcommand\\(chkSolv\w+)\{([^}]*)\}", checks))
solv_src = (ROOT / "docs/techref/figures/solvers.jl").read_text()
for needle in ("const SOLV_RTOL = 1.0e-10", "const SOLV_DENSITY = (1000.0, 1.0)",
               "SOLV_DROP = (; centre = (0.513, 0.468), radius = 0.2371, band = 0.02)",
               "solv_noise(index) = (value = sin(12.9898 * index) * 43758.5453; value - floor(value) - 0.5)",
               "base_mesh = (n, n), block_size = (8, 8), periodic = (false, false)"):
    assert needle in solv_src, needle
cases = {}
for key, name in (("UniformA", "uniform64"), ("UniformB", "uniform128"), ("UniformC", "uniform256"),
                  ("AmrA", "amr32"), ("AmrB", "amr64"), ("Drop", "drop128"), ("DropAmr", "dropamr")):
    cases[name] = {"unknowns": int(macros[f"chkSolv{key}Unknowns"]), "levels": int(macros[f"chkSolv{key}Levels"]),
                   "cycles": int(macros[f"chkSolv{key}Cycles"]), "factor": macros[f"chkSolv{key}Factor"],
                   "plain_cycles": int(macros[f"chkSolv{key}Plain"])}
vcycle = {"uniform16": {"kappa": macros["chkSolvKappaUniformA"]},
          "uniform32": {"kappa": macros["chkSolvKappaUniformB"], "bound": macros["chkSolvBoundUniform"],
                        "cycles": int(macros["chkSolvCgUniform"]), "factor": macros["chkSolvCgUniformFactor"]},
          "amr16": {"kappa": macros["chkSolvKappaAmr"], "cells": int(macros["chkSolvVcycleCells"])},
          "drop32": {"kappa": macros["chkSolvKappaDrop"], "bound": macros["chkSolvBoundDrop"],
                     "cycles": int(macros["chkSolvCgDrop"]), "factor": macros["chkSolvCgDropFactor"]}}
out["techref_pressure_solves"] = {
    "source": "docs/techref/figures/generated/checks.tex (chkSolv* macros) written by "
              "docs/techref/figures/solvers.jl:72-165, 425-525",
    "fixture": "walls (periodic false), block 8x8; uniform n: base_mesh (n, n); amr n: base (n, n), max_level 2, "
               "refine blocks whose box comes within 0.02 of the circle centre (0.513, 0.468), radius 0.2371; "
               "drop: fractions of that circle (liquid inside), density (1000, 1); RHS solv_noise(cell index), "
               "rtol 1e-10, default MultigridOptions",
    "solves": cases, "vcycle": vcycle,
    "lambda_min_all": macros["chkSolvLambdaMin"], "lambda_max_all": macros["chkSolvLambdaMax"],
    "omega_uniform128": macros["chkSolvOmegaUniform"], "omega_amr64": macros["chkSolvOmegaAmr"],
    "omega_drop128": macros["chkSolvOmegaDrop"],
}
(pathlib.Path(__file__).parent / "known_answers.json").write_text(json.dumps(out, indent=1))
print("wrote", len(rows), "table rows")
