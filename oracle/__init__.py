"""CPU oracle and reference-engine shim for the GPU dictionary.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
(and its ``--impl reference`` arm) may import this package.  The product path in
``gpu-lsm-tree_b200/`` never calls it and has no CPU fallback.
"""
from .oracle import CpuLsm, CpuMap, OracleLSM, OracleFlix, oracle_threads, build_oracle  # noqa: F401
