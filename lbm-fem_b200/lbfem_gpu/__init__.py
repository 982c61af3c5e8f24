"""Host side of the B200 implementation of lbm-fem's per-time-step hot path.

The compute lives in the CUDA library ``liblbfem_gpu.so`` (sources in
``../csrc``, C ABI in ``include/lbfem_gpu.h``); this package binds it with
ctypes and mirrors the reference's host interface:

* ``Solver`` -- one context: Scheme::set_time_step / set_initial_populations /
  step (schemes.h), AdvectionOperator::apply (advection.h), MassSolver::solve
  (mass.h), collide_bgk / compute_equilibrium / predictor_corrector
  (collision.h), node_weight (discretization.h).
* ``cases`` -- the TestCase flows and the tensor-product mesh export.

The library must be built (``__graft_entry__.build()`` or ``make -C csrc``);
there is no CPU fallback: without the library or a GPU, ``Solver`` raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import cases, d2q9
from ._abi import LbfemError, NoConvergence, make_params

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "liblbfem_gpu.so")

_lib = None


def library():
    """The loaded CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LbfemError(4, f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
        from . import _abi

        lib = C.CDLL(LIB_PATH)
        _abi.declare(lib, "lbfem_gpu_")
        lib.lbfem_gpu_last_error.restype = C.c_char_p
        lib.lbfem_gpu_last_error.argtypes = [C.c_void_p]
        lib.lbfem_gpu_device_count.restype = C.c_int
        lib.lbfem_gpu_device_count.argtypes = []
        lib.lbfem_gpu_host_alloc.restype = C.c_void_p
        lib.lbfem_gpu_host_alloc.argtypes = [C.c_size_t]
        lib.lbfem_gpu_host_free.restype = None
        lib.lbfem_gpu_host_free.argtypes = [C.c_void_p]
        lib.lbfem_gpu_status_string.restype = C.c_char_p
        lib.lbfem_gpu_status_string.argtypes = [C.c_int]
        _lib = lib
    return _lib


def device_count():
    return library().lbfem_gpu_device_count()


class Solver:
    """A context of the CUDA library; same methods as the oracle's handle."""

    def __new__(cls, mesh, params, dof_index=None):
        from ._abi import Handle

        return Handle(library(), "lbfem_gpu_", mesh, params, dof_index=dof_index)


class Batch:
    """Independent instances (Solver handles on one device) stepped together:
    each step of all of them is one graph launch (lbfem_gpu_batch_step). The
    handles stay usable on their own; keep them alive while the batch is."""

    def __init__(self, solvers):
        from ._abi import LbfemError

        self.lib = library()
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s.h.value for s in self.solvers])
        fn = self.lib.lbfem_gpu_batch_create
        fn.restype, fn.argtypes = C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]
        h = C.c_void_p()
        st = fn(arr, len(self.solvers), C.byref(h))
        if st != 0:
            raise LbfemError(st, "lbfem_gpu_batch_create")
        self.h = h
        self.lib.lbfem_gpu_batch_last_error.restype = C.c_char_p
        self.lib.lbfem_gpu_batch_last_error.argtypes = [C.c_void_p]

    def step(self, n=1):
        from ._abi import LBFEM_ERR_NO_CONVERGENCE, LbfemError, NoConvergence

        fn = self.lib.lbfem_gpu_batch_step
        fn.restype, fn.argtypes = C.c_int, [C.c_void_p, C.c_int32]
        st = fn(self.h, int(n))
        if st != 0:
            msg = self.lib.lbfem_gpu_batch_last_error(self.h).decode()
            raise (NoConvergence if st == LBFEM_ERR_NO_CONVERGENCE else LbfemError)(st, f"lbfem_gpu_batch_step: {msg}")

    def last_ms(self):
        """Device time (CUDA events on the batch stream) of the last step call's launches."""
        fn = self.lib.lbfem_gpu_batch_last_ms
        fn.restype, fn.argtypes = C.c_int, [C.c_void_p, C.POINTER(C.c_float)]
        ms = C.c_float()
        fn(self.h, C.byref(ms))
        return ms.value

    def last_launches(self):
        """Kernels launched by the last step call (all instances and the grouped launches)."""
        fn = self.lib.lbfem_gpu_batch_last_launches
        fn.restype, fn.argtypes = C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]
        n = C.c_int64()
        fn(self.h, C.byref(n))
        return int(n.value)

    def close(self):
        if getattr(self, "h", None) is not None:
            fn = self.lib.lbfem_gpu_batch_destroy
            fn.restype, fn.argtypes = C.c_int, [C.c_void_p]
            fn(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["Solver", "Batch", "cases", "d2q9", "make_params", "LbfemError", "NoConvergence", "library",
           "device_count"]
