"""qikkdb_b200: the GROUP BY hot path of qikkDB (filter -> compaction -> hash aggregation) rebuilt as
hand-written sm_100a CUDA kernels behind a C ABI (include/qdb_gb.h), with a Python mirror of the
reference's operator classes for tests and benchmarks.

The CUDA library is loaded lazily by ``qikkdb_b200._capi.lib()``; it must have been built in-tree
(``python -m qikkdb_b200.build``).  There is no CPU execution path.
"""
from . import _capi  # noqa: F401

__all__ = ["_capi"]
__version__ = "0.1.0"
