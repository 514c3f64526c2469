"""CPU oracle for the exFEMuS assembly + multigrid path (test infrastructure only).

This package is the checker: tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg call it.  The product library never imports it.

`Oracle*` classes wrap liboracle.so (oracle.c, a restatement of the reference's
C++ layer); `Laspack` wraps _ref/liblaspack_ref.so, the reference's vendored
LASPACK C library compiled from its own sources (absent when the reference tree was
not available at build time).
"""
from .pyoracle import (OrMesh, OrSys, OrPhys, OrMgParams, OrMgStats, Laspack, build,  # noqa: F401
                       laspack_available, oracle_lib, set_threads, get_threads)
