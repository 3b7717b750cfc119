"""everest_b200 -- a B200-native (sm_100a) temporal-motif miner.

Drop-in for the hot path of Everest: per-motif backtracking search (count and
enumerate) over a time-sorted temporal edge list, behind the reference's
query surface (YAML queries, the ``corelib`` pybind11 module, the
``getWorker`` plugin ABI).  The compute path is hand-written CUDA for
sm_100a behind the C ABI in ``include/everest_b200.h``.
"""
__version__ = "0.1.0"
