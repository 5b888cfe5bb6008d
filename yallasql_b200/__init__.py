"""yallasql_b200 — B200-native (sm_100a) per-batch SQL operators.

Drop-in for YallaSQL's kernel layer: the CUDA kernels and their C ABI live in
``libyq_ops.so`` (``include/yq_ops.h``); the C++ operator layer mirroring the
reference's pull-based operator API lives in ``libyq_engine.so``
(``include/yq_engine.h``). This package holds the build script, ctypes
bindings, the expression compiler and torch-facing wrappers used by tests and
the benchmark.
"""
from . import _abi  # noqa: F401
from ._abi import YQError  # noqa: F401

__all__ = ["_abi", "YQError", "load"]


def load():
    """Load libyq_ops.so (raises ImportError when it has not been built)."""
    return _abi.load()
