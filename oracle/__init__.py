"""CPU FP64 oracle for llg-sim's uniform-grid LLG hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker.  The product library
(llg-sim_b200/) never imports, links or calls anything in this package.

The C++ restatement lives in oracle.cpp (built into liboracle.so by the
Makefile); this module wraps it with ctypes and numpy.  Arrays are numpy
float64 in the reference's layout: AoS ``[nx*ny, 3]`` with ``idx = j*nx + i``
(grid.rs:27-30, vector_field.rs:24-27).
"""
from .oracle import *  # noqa: F401,F403
