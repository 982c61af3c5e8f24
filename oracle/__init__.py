"""ctypes binding of the CPU FP64 oracle (oracle/lbfem_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker of the CUDA path. The product
package never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblbfem_oracle.so")
REF_STENCIL_BENCH = os.path.join(HERE, "_ref", "stencil_bench")

_lib = None


def build(force=False):
    """Builds the oracle library with the Makefile in this directory."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "oracle"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        from lbfem_gpu import _abi

        _lib = _abi.declare(C.CDLL(LIB_PATH), "lbfem_oracle_")
        _lib.lbfem_oracle_set_threads.restype = C.c_int
        _lib.lbfem_oracle_set_threads.argtypes = [C.c_int32]
        _lib.lbfem_oracle_basis_1d.restype = C.c_int
        _lib.lbfem_oracle_basis_1d.argtypes = [C.c_int32] + [C.POINTER(C.c_double)] * 3
    return _lib


def set_threads(n):
    """OpenMP threads of the oracle (n <= 0 keeps the current number); returns the number in use."""
    return lib().lbfem_oracle_set_threads(n)


def basis_1d(p):
    import numpy as np

    s, g, w = np.empty(p + 1), np.empty(p + 1), np.empty(p + 1)
    P = C.POINTER(C.c_double)
    st = lib().lbfem_oracle_basis_1d(p, s.ctypes.data_as(P), g.ctypes.data_as(P), w.ctypes.data_as(P))
    assert st == 0
    return s, g, w


def Oracle(mesh, params):
    """A context of the oracle with the same methods as the CUDA library's (lbfem_gpu._abi.Handle)."""
    from lbfem_gpu import _abi

    return _abi.Handle(lib(), "lbfem_oracle_", mesh, params)
