"""CPU oracle for the pressure-projection solve of TwoPhaseAMR.jl.

TEST INFRASTRUCTURE ONLY.  This package restates the reference's algorithm on
the CPU (numpy/scipy, plus a C/OpenMP restatement of the solve loop in
`cgmg.c`) so that tests can check the B200 library against it.  Only `tests/`,
`__graft_entry__.smoke()` and the CPU-baseline leg of `bench.py` may import or
run anything here; the shipped solver never does.

Parity pinning: the reference is Julia and cannot run in this container, so
this restatement is pinned against the reference's own published known
answers (see `tests/golden/` and `tests/test_oracle_golden.py`): the PCG
iteration counts and discretisation errors of `docs/src/poisson.md:253-257`
(test `test/operators/poisson.jl:728-831`), the hierarchy sizes of
`test/operators/poisson.jl:422-611`, and the Jacobi-weight values of
`test/operators/poisson.jl:300-317`.
"""
