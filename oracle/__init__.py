"""ORACLE — test infrastructure only (the checker, never the product).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg and
reference arm import this package.  It binds three libraries built by
oracle/Makefile:

* liboracle.so — oracle.c, a plain-C restatement of the reference's CPU SpMV
  path and format converters;
* _ref/libmfp_ref.so — the reference's own sources (common/, cpu/,
  gpu/csr_adaptive_spmv.cu) compiled unmodified, when the reference checkout
  was available at build time;
* libmfp_synth.so — the seeded matrix generator alone (the engine's
  csrc/synth.cpp built without the engine), so that the benchmark's
  reference arm generates its matrix without mapping the engine's library.

The restatement is pinned to the reference by tests/test_oracle.py (against
_ref when present, and always against the committed fixtures in
tests/golden/, which _ref produced).
"""
from .oracle import (HERE, Oracle, RefLib, build, load_oracle, load_ref, load_synth, synth_power_law)  # noqa: F401
