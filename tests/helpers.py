"""Shared set-up for the tests: meshes, runs of a case on a backend, errors."""
import math

import numpy as np

from lbfem_gpu import cases, d2q9, make_params


def unit_mesh(n, p, periodic=(True, True), h=1.0, ny=None):
    """A uniform n x ny mesh of cells of size h (periodic by default), no walls."""
    ny = n if ny is None else ny
    return cases.Mesh(p, n, ny, periodic[0], periodic[1], np.arange(n + 1) * h, np.arange(ny + 1) * h, h)


def setup_case(backend, tc, mesh, params, dt, lam):
    h = backend(mesh, params)
    h.set_time_step(dt, lam)
    x, y = mesh.nodes()
    h.set_initial_populations(tc.initial_populations(x, y, lam))
    return h


def tgv(N, p=1, mach=0.05, Re=100, modes=(1, 4), **kw):
    tc = cases.TaylorGreenVortex(mach, *modes, **kw)
    tc.set_reynolds(Re)
    return tc, cases.build_mesh(tc, N, p)


def rel_l2(a, b, mask=None):
    if mask is not None:
        a, b = a[..., mask], b[..., mask]
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def directions():
    return np.ascontiguousarray(d2q9.E, dtype=np.float64)


def random_populations(mesh, seed=0, amp=1e-2, u0=0.05):
    """Smooth-ish positive populations around a random flow: feq(rho, u) + noise."""
    rng = np.random.default_rng(seed)
    x, y = mesh.nodes()
    rho = 1.0 + 0.01 * np.sin(2 * math.pi * x) * np.cos(2 * math.pi * y) + 0.001 * rng.standard_normal(x.shape)
    ux = u0 * np.sin(2 * math.pi * y) + 0.001 * rng.standard_normal(x.shape)
    uy = -u0 * np.cos(2 * math.pi * x) + 0.001 * rng.standard_normal(x.shape)
    f = d2q9.equilibrium(rho, ux, uy)
    f += amp * 1e-2 * rng.standard_normal(f.shape)
    # periodic images carry their source's value, as after constraints.distribute
    return f[:, mesh.master()]
