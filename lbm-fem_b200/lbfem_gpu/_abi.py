"""ctypes view of the C ABI in include/lbfem_gpu.h: the two structs, the status
codes, and a thin object wrapper whose methods mirror the reference's
operator interface (Scheme, AdvectionOperator, MassSolver, the nodal
functions of collision.h). Errors come back as LbfemError, the analogue of the
reference's exceptions (AssertThrow, SolverControl::NoConvergence)."""
from __future__ import annotations

import ctypes as C

import numpy as np

LBFEM_OK = 0
LBFEM_ERR_ARG = 1
LBFEM_ERR_NO_CONVERGENCE = 2
LBFEM_ERR_NONFINITE = 3
LBFEM_ERR_CUDA = 4
LBFEM_ERR_UNSUPPORTED = 5
LBFEM_ERR_TIMEOUT = 6
LBFEM_ERR_STATE = 7

SCHEME = {"leelin": 0, "bardow": 1}
MASS = {"cg": 0, "lumped": 1, "richardson": 2}
PRECISION = {"fp64": 0, "mixed": 1}
ADVECTION = {"taylor_galerkin": 0, "leelin": 1}
STREAMING = {"tg2": 0, "tg3": 1, "tg3-split": 2}

_STATUS = {
    0: "ok", 1: "bad argument", 2: "CG did not converge", 3: "non-finite value",
    4: "CUDA error", 5: "unsupported", 6: "device wait timed out", 7: "call out of order",
}


class LbfemError(RuntimeError):
    def __init__(self, status, message=""):
        self.status = status
        super().__init__(f"{_STATUS.get(status, status)} ({status}){': ' + message if message else ''}")


class NoConvergence(LbfemError):
    """SolverControl::NoConvergence of the reference (mass.h:38-43)."""


class MeshDesc(C.Structure):
    _fields_ = [
        ("degree", C.c_int32), ("n_cells_x", C.c_int32), ("n_cells_y", C.c_int32),
        ("periodic_x", C.c_int32), ("periodic_y", C.c_int32),
        ("vertex_x", C.POINTER(C.c_double)), ("vertex_y", C.POINTER(C.c_double)),
        ("n_dofs", C.c_int64), ("dof_index", C.POINTER(C.c_int64)),
        ("n_walls", C.c_int64), ("wall_dof", C.POINTER(C.c_int64)), ("wall_velocity", C.POINTER(C.c_double)),
        ("vertex_xy", C.POINTER(C.c_double)),
    ]


class Params(C.Structure):
    _fields_ = [
        ("scheme", C.c_int32), ("mass", C.c_int32), ("richardson", C.c_int32), ("streaming", C.c_int32),
        ("precision", C.c_int32), ("cg_max_iterations", C.c_int32), ("cg_tolerance", C.c_double),
        ("remove_wall_mass_flux", C.c_int32), ("device", C.c_int32), ("mixed_tolerance", C.c_double),
    ]


def make_params(scheme="bardow", mass="cg", cg_tolerance=1e-8, cg_max_iterations=200, precision="fp64",
                richardson=2, remove_wall_mass_flux=-1, device=0, mixed_tolerance=0.0, streaming="tg2"):
    return Params(SCHEME[scheme], MASS[mass], richardson, STREAMING[streaming], PRECISION[precision],
                  cg_max_iterations, cg_tolerance, remove_wall_mass_flux, device, mixed_tolerance)


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Handle:
    """One context of a library that implements the C ABI under ``prefix``
    (``lbfem_gpu_`` for the CUDA library, ``lbfem_oracle_`` for the CPU oracle)."""

    def __init__(self, lib, prefix, mesh, params, dof_index=None):
        self.lib, self.prefix, self.mesh = lib, prefix, mesh
        self.n = mesh.n_dofs
        self._keep = [np.ascontiguousarray(mesh.vertex_x, np.float64), np.ascontiguousarray(mesh.vertex_y, np.float64),
                      np.ascontiguousarray(mesh.wall_dof, np.int64),
                      np.ascontiguousarray(mesh.wall_velocity, np.float64).reshape(-1)]
        di = None
        if dof_index is not None:
            di = np.ascontiguousarray(dof_index, np.int64)
            self._keep.append(di)
        vxy = None
        if getattr(mesh, "vertex_xy", None) is not None:
            vxy = np.ascontiguousarray(mesh.vertex_xy, np.float64).reshape(-1)
            self._keep.append(vxy)
        desc = MeshDesc(mesh.degree, mesh.n_cells_x, mesh.n_cells_y, int(mesh.periodic_x), int(mesh.periodic_y),
                        _dptr(self._keep[0]), _dptr(self._keep[1]), mesh.n_dofs,
                        di.ctypes.data_as(C.POINTER(C.c_int64)) if di is not None else None,
                        len(self._keep[2]), self._keep[2].ctypes.data_as(C.POINTER(C.c_int64)),
                        _dptr(self._keep[3]), _dptr(vxy))
        self.params = params
        h = C.c_void_p()
        self._call("create", C.byref(desc), C.byref(params), C.byref(h))
        self.h = h

    # -- plumbing
    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def _call(self, name, *args):
        st = self._fn(name)(*args)
        if st != LBFEM_OK:
            msg = ""
            if self.prefix == "lbfem_gpu_" and getattr(self, "h", None) is not None:
                msg = self.lib.lbfem_gpu_last_error(self.h).decode()
            cls = NoConvergence if st == LBFEM_ERR_NO_CONVERGENCE else LbfemError
            raise cls(st, f"{self.prefix}{name}" + (f": {msg}" if msg else ""))
        return st

    def close(self):
        if getattr(self, "h", None) is not None:
            self._fn("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- Scheme
    def set_time_step(self, dt, lam):
        self._call("set_time_step", self.h, C.c_double(dt), C.c_double(lam))

    def set_initial_populations(self, f):
        f = _f64(f)
        self._call("set_initial_populations", self.h, _dptr(f))

    def set_populations(self, f):
        f = _f64(f)
        self._call("set_populations", self.h, _dptr(f))

    def get_populations(self):
        out = np.empty((9, self.n))
        self._call("get_populations", self.h, _dptr(out))
        return out

    def write_checkpoint(self, name, rank=0):
        """write_checkpoint (io.h:144-154): the raw populations to name.rank."""
        self._call("write_checkpoint", self.h, str(name).encode(), C.c_int32(rank))

    def read_checkpoint(self, name, rank=0):
        """read_checkpoint (io.h:156-165)."""
        self._call("read_checkpoint", self.h, str(name).encode(), C.c_int32(rank))

    def step(self, n=1):
        self._call("step", self.h, C.c_int32(n))

    # -- operators
    def advection(self, f, e, dt, lam, kind="taylor_galerkin", feq=None, remove_wall_mass_flux=-1):
        f, e = _f64(f), _f64(e)
        feq = _f64(feq) if feq is not None else None
        rhs = np.empty((8, self.n))
        self._call("advection", self.h, _dptr(f), _dptr(feq), _dptr(e), C.c_double(dt), C.c_double(lam),
                   C.c_int32(ADVECTION[kind]), C.c_int32(remove_wall_mass_flux), _dptr(rhs))
        return rhs

    def mass_solve(self, r, x=None, e=(0.0, 0.0), tg3_coefficient=0.0):
        r = _f64(r)
        x = np.zeros(self.n) if x is None else _f64(x).copy()
        e = _f64(e)
        self._call("mass_solve", self.h, _dptr(x), _dptr(r), _dptr(e), C.c_double(tg3_coefficient))
        return x

    def stream_function(self, velocity):
        """compute_stream_function (io.h:31-95): psi from velocity = (u, v) (2 x n_dofs)."""
        velocity = _f64(velocity).reshape(2, self.n)
        psi = np.empty(self.n)
        self._call("stream_function", self.h, _dptr(velocity), _dptr(psi))
        return psi

    def mass_vmult(self, x):
        x = _f64(x)
        y = np.empty(self.n)
        self._call("mass_vmult", self.h, _dptr(y), _dptr(x))
        return y

    def cg_iterations(self):
        v = C.c_int64()
        self._call("cg_iterations", self.h, C.byref(v))
        return v.value

    def collide_bgk(self, g, omega):
        g = _f64(g).copy()
        self._call("collide_bgk", self.h, _dptr(g), C.c_double(omega))
        return g

    def compute_equilibrium(self, f):
        f = _f64(f)
        out = np.empty((9, self.n))
        self._call("compute_equilibrium", self.h, _dptr(f), _dptr(out))
        return out

    def predictor_corrector(self, f, feq, incr, theta):
        f = _f64(f).copy()
        feq, incr = _f64(feq), _f64(incr)
        self._call("predictor_corrector", self.h, _dptr(f), _dptr(feq), _dptr(incr), C.c_double(theta))
        return f

    # -- device-pointer forms: arguments are device addresses (ints) and the
    #    caller's cudaStream_t as an int (0: the legacy default stream)
    def advection_dev(self, f, e, dt, lam, rhs, kind="taylor_galerkin", feq=0, remove_wall_mass_flux=-1, stream=0):
        e = _f64(e)
        self._call("advection_dev", self.h, f, feq or None, _dptr(e), C.c_double(dt), C.c_double(lam),
                   C.c_int32(ADVECTION[kind]), C.c_int32(remove_wall_mass_flux), rhs, stream or None)

    def mass_solve_dev(self, x, r, e=(0.0, 0.0), tg3_coefficient=0.0, stream=0):
        e = _f64(e)
        self._call("mass_solve_dev", self.h, x, r, _dptr(e), C.c_double(tg3_coefficient), stream or None)

    def collide_bgk_dev(self, g, omega, stream=0):
        self._call("collide_bgk_dev", self.h, g, C.c_double(omega), stream or None)

    def compute_equilibrium_dev(self, f, feq, stream=0):
        self._call("compute_equilibrium_dev", self.h, f, feq, stream or None)

    def predictor_corrector_dev(self, f, feq, incr, theta, stream=0):
        self._call("predictor_corrector_dev", self.h, f, feq, incr, C.c_double(theta), stream or None)

    def set_populations_dev(self, f, stream=0):
        self._call("set_populations_dev", self.h, f, stream or None)

    def get_populations_dev(self, f, stream=0):
        self._call("get_populations_dev", self.h, f, stream or None)

    def step_stream(self, n=1, stream=0):
        self._call("step_stream", self.h, C.c_int32(n), stream or None)

    def node_weight(self):
        w = np.empty(self.n)
        self._call("node_weight", self.h, _dptr(w))
        return w

    def jacobi_diagonal(self):
        d = np.empty(self.n)
        self._call("jacobi_diagonal", self.h, _dptr(d))
        return d

    def conservation(self):
        out = np.empty(5)
        self._call("conservation", self.h, _dptr(out))
        return out


def declare(lib, prefix):
    """Sets restype/argtypes of the ABI functions that exist in lib."""
    vp, i32, i64, d, dp = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.POINTER(C.c_double)
    sig = {
        "create": [C.POINTER(MeshDesc), C.POINTER(Params), C.POINTER(vp)],
        "destroy": [vp], "set_time_step": [vp, d, d], "set_initial_populations": [vp, dp],
        "set_populations": [vp, dp], "get_populations": [vp, dp], "step": [vp, i32],
        "step_host": [vp, dp, i32], "synchronize": [vp],
        "advection": [vp, dp, dp, dp, d, d, i32, i32, dp],
        "mass_solve": [vp, dp, dp, dp, d], "mass_vmult": [vp, dp, dp], "stream_function": [vp, dp, dp],
        "cg_iterations": [vp, C.POINTER(i64)], "collide_bgk": [vp, dp, d],
        "compute_equilibrium": [vp, dp, dp], "predictor_corrector": [vp, dp, dp, dp, d],
        "node_weight": [vp, dp], "jacobi_diagonal": [vp, dp], "conservation": [vp, dp],
        "moments": [vp, dp, dp, dp], "event_record": [vp, i32],
        "event_elapsed": [vp, i32, i32, C.POINTER(C.c_float)], "advection_resident": [vp],
        "solve_round_resident": [vp],
        "last_step_stats": [vp, dp, C.POINTER(i64)],
        "write_checkpoint": [vp, C.c_char_p, i32], "read_checkpoint": [vp, C.c_char_p, i32],
        # device-pointer forms (vp: device addresses and the caller's cudaStream_t)
        "advection_dev": [vp, vp, vp, dp, d, d, i32, i32, vp, vp],
        "mass_solve_dev": [vp, vp, vp, dp, d, vp], "collide_bgk_dev": [vp, vp, d, vp],
        "compute_equilibrium_dev": [vp, vp, vp, vp], "predictor_corrector_dev": [vp, vp, vp, vp, d, vp],
        "set_populations_dev": [vp, vp, vp], "get_populations_dev": [vp, vp, vp], "step_stream": [vp, i32, vp],
        # y-strip decomposition (strips.py)
        "strip_buffer_bytes": [vp, C.POINTER(i64)], "set_strip": [vp, vp],
        "tuning": [vp, C.POINTER(i32), C.POINTER(C.c_float)],
    }
    for name, args in sig.items():
        fn = getattr(lib, prefix + name, None)
        if fn is not None:
            fn.restype = C.c_int
            fn.argtypes = args
    return lib
