"""CPU oracle for the SpecAnn alpha-sweep hot path.

TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
(and its ``--impl reference`` arm) may import anything here, and only as the checker or the timed
CPU baseline. The product (specann_b200) never imports, links or calls this package: it has no CPU
fallback.

Modules:
  specann_oracle  NumPy/SciPy restatement of the reference solver (prelude, schedule, operators,
                  shift, predictors, eigensolve with retry/checks, rounding, signatures, energies,
                  local search, best-candidate selection), the reference kernel's in-order fp32 pass
                  and the deviation count against it, and row-block threaded products for the timed
                  CPU baseline.
  selection       the counter-based node-selection stream shared with the CUDA local search.
  guards_oracle   the guarded local-search policies (fixed / adaptive guard, independent set,
                  sequential oracle).
  adjoint_oracle  dense FP64 eigenvector adjoint and gradient (the differentiation form's checker).
  build_tools     builds _bin/ba_graph from ba_graph_main.cpp: the stand-alone graph writer the CPU
                  reference arm runs, so that its process loads none of the product's libraries.

Parity pin: tests/golden/make_golden.py runs the reference's own solver code (the CuPy files of the
reference, executed on NumPy/SciPy through a stand-in module) and freezes its per-alpha records;
tests/test_oracle_golden.py checks this oracle against them.
"""
