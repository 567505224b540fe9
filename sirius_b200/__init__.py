"""sirius_b200 — a B200-native (sm_100a) equi-hash-join for Sirius's physical hash-join operator.

The join itself lives in ``libsj.so`` (hand-written CUDA behind the C ABI of
``include/sj/sj_join.h``); this package holds its build recipe, the torch-facing host API and the
synthetic workload generators.
"""
__all__ = ["join", "datagen", "build"]
