"""Host-side set-up of the flows and meshes the hot path runs on: the
TestCase interface and the three benchmark flows of include/lbfem/test_case.h
and test_cases.h, the tensor-product mesh of Discretization::reinit
(discretization.h:78-144) and the driver's time-step rule (cgdbe.cc:233-242).

Everything here runs once per run on the host; it produces the flat arrays of
an ``lbfem_mesh_desc`` (vertex coordinates per axis, periodicity, wall nodes
and velocities) and the initial populations.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import d2q9


def gauss_lobatto(p: int) -> np.ndarray:
    """FE_Q(p) support points on [0, 1]: the Gauss-Lobatto points."""
    if p == 1:
        return np.array([0.0, 1.0])
    inner = np.polynomial.legendre.Legendre.basis(p).deriv().roots()
    t = np.concatenate([[-1.0], np.sort(inner.real), [1.0]])
    return (t + 1.0) / 2.0


# --------------------------------------------------------------- test cases
class TestCase:
    """test_case.h:23-83. Lattice units; U0 = Ma c_s; nu = U0 L / Re; lambda = nu / c_s^2."""

    L = 1.0
    rho0 = 1.0

    def __init__(self, mach: float):
        self.U0 = mach * math.sqrt(d2q9.CS2)
        self.nu = 0.0

    def set_reynolds(self, Re: float):
        self.nu = self.U0 * self.L / Re

    def relaxation_time(self) -> float:
        return self.nu / d2q9.CS2

    n_periodic = 0
    steady = False

    def reference_time(self) -> float:
        raise NotImplementedError

    def transform_axes(self, vx, vy, h_min):
        return vx, vy, h_min

    def wall_velocity(self, x, y):
        """(mask, ux, uy) arrays: which nodes are wall nodes and their wall velocity."""
        z = np.zeros_like(x)
        return np.zeros(x.shape, bool), z, z

    def exact(self, x, y, t):
        return np.full_like(x, self.rho0), np.zeros_like(x), np.zeros_like(x)

    def energy_scale(self) -> float:
        return self.U0 * self.U0

    def initial_populations(self, x, y, lam):
        rho, ux, uy = self.exact(x, y, 0.0)
        return d2q9.equilibrium(rho, ux, uy)


class TaylorGreenVortex(TestCase):
    """test_cases.h:105-203 (Bardow et al., Eqs. (14)-(16)), with wave numbers k_i = 2 pi n_i / L.

    ``shift`` translates the vortex by (sx, sy) (the solution at x + shift), and
    ``chapman_enskog=False`` starts from f = feq without the first-order
    Chapman-Enskog part; shift (L/4, L/4) gives u = U0 sin(2 pi x) cos(2 pi y),
    v = -U0 cos(2 pi x) sin(2 pi y) for modes (1, 1)."""

    n_periodic = 2
    steady = False

    def __init__(self, mach, n1=1, n2=4, shift=(0.0, 0.0), chapman_enskog=True, distort=0.0):
        super().__init__(mach)
        self.n1, self.n2 = float(n1), float(n2)
        self.shift = shift
        self.chapman_enskog = chapman_enskog
        self.distort = float(distort)

    def transform_vertices(self, X, Y):
        """TaylorGreenVortex::transform_mesh (test_cases.h:52-63): every vertex moves by
        eps L sin(2 pi x / L) sin(2 pi y / L) (1, 1) (zero on the box's sides, so the
        periodic sides still match); the cells become general quadrilaterals."""
        d = self.distort * self.L * np.sin(2 * math.pi * X / self.L) * np.sin(2 * math.pi * Y / self.L)
        return X + d, Y + d

    def k1(self):
        return 2 * math.pi * self.n1 / self.L

    def k2(self):
        return 2 * math.pi * self.n2 / self.L

    def decay(self, t):
        return math.exp(-self.nu * (self.k1() ** 2 + self.k2() ** 2) * t)

    def reference_time(self):
        return 1.0 / (self.nu * (self.k1() ** 2 + self.k2() ** 2))

    def energy_scale(self):
        r = self.k1() / self.k2()
        return 0.25 * self.U0 * self.U0 * (1 + r * r)

    def exact(self, x, y, t):
        x = x + self.shift[0]
        y = y + self.shift[1]
        F = self.decay(t)
        x1, y2, r = self.k1() * x, self.k2() * y, self.k1() / self.k2()
        dp = -0.25 * self.rho0 * self.U0 ** 2 * F * F * (np.cos(2 * x1) + r * r * np.cos(2 * y2))
        return (self.rho0 + dp / d2q9.CS2, -self.U0 * F * np.cos(x1) * np.sin(y2),
                self.U0 * r * F * np.sin(x1) * np.cos(y2))

    def initial_populations(self, x, y, lam):
        rho, ux, uy = self.exact(x, y, 0.0)
        f = d2q9.equilibrium(rho, ux, uy)
        if not self.chapman_enskog:
            return f
        xs, ys = x + self.shift[0], y + self.shift[1]
        x1, y2 = self.k1() * xs, self.k2() * ys
        dudx = self.U0 * self.k1() * np.sin(x1) * np.sin(y2)
        shear = self.U0 * (self.k1() ** 2 - self.k2() ** 2) / self.k2() * np.cos(x1) * np.cos(y2)
        for a in range(d2q9.Q):
            ex, ey = d2q9.E[a]
            f[a] -= lam / d2q9.CS2 * d2q9.W[a] * rho * ((ex * ex - ey * ey) * dudx + ex * ey * shear)
        return f


class CouetteFlow(TestCase):
    """test_cases.h:209-264: start-up Couette flow, periodic in x, bottom wall at rest, top wall at U0."""

    n_periodic = 1
    steady = False

    def reference_time(self):
        return self.L * self.L / self.nu

    def wall_velocity(self, x, y):
        bottom = np.abs(y) < 1e-12 * self.L
        top = np.abs(y - self.L) < 1e-12 * self.L
        ux = np.where(top, self.U0, 0.0)
        return bottom | top, ux, np.zeros_like(x)

    def exact(self, x, y, t):
        u = self.U0 * y / self.L
        for m in range(1, 401):
            lm = m * math.pi / self.L
            u = u + 2.0 * self.U0 * (-1.0 if m % 2 else 1.0) / (lm * self.L) * math.exp(-self.nu * lm * lm * t) * np.sin(lm * y)
        return np.full_like(x, self.rho0), u, np.zeros_like(x)

    def initial_populations(self, x, y, lam):
        one = np.ones_like(x)
        return d2q9.equilibrium(self.rho0 * one, 0 * one, 0 * one)


class LidDrivenCavity(TestCase):
    """test_cases.h:270-329: tanh-clustered mesh, walls at rest, lid at U0 (top corners at rest)."""

    n_periodic = 0
    steady = True

    def __init__(self, mach, stretch=1.2):
        super().__init__(mach)
        self.stretch = stretch

    def reference_time(self):
        return self.L / self.U0

    def cluster(self, x):
        s = self.stretch
        return 0.5 * self.L * (1.0 + np.tanh(s * (2.0 * x / self.L - 1.0)) / math.tanh(s))

    def transform_axes(self, vx, vy, h_min):
        if self.stretch <= 0:
            return vx, vy, h_min
        return self.cluster(vx), self.cluster(vy), float(self.cluster(h_min))

    def wall_velocity(self, x, y):
        on = lambda a, a0: np.abs(a - a0) < 1e-12 * self.L
        still = on(x, 0.0) | on(x, self.L) | on(y, 0.0)
        lid = on(y, self.L) & ~still
        return still | lid, np.where(lid, self.U0, 0.0), np.zeros_like(x)


# ---------------------------------------------------------------- the mesh
@dataclass
class Mesh:
    """A structured tensor-product discretisation (discretization.h:78-144)."""

    degree: int
    n_cells_x: int
    n_cells_y: int
    periodic_x: bool
    periodic_y: bool
    vertex_x: np.ndarray
    vertex_y: np.ndarray
    h_min: float
    wall_dof: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    wall_velocity: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))
    # mapped vertices ((n_cells_y + 1) x (n_cells_x + 1) x 2) of a general quadrilateral mesh, or None
    vertex_xy: np.ndarray | None = None

    @property
    def nfx(self):
        return self.degree * self.n_cells_x + 1

    @property
    def nfy(self):
        return self.degree * self.n_cells_y + 1

    @property
    def n_dofs(self):
        return self.nfx * self.nfy

    def axis_nodes(self, v):
        xi = gauss_lobatto(self.degree)
        h = np.diff(v)
        pts = (v[:-1, None] + h[:, None] * xi[None, :-1]).ravel()
        return np.concatenate([pts, v[-1:]])

    def nodes(self):
        """Support points (x, y) of all structured nodes, node (i, j) at j*nfx + i. On a
        general quadrilateral mesh: the bilinear image (MappingQ1) of each node's
        Gauss-Lobatto point in its cell."""
        if self.vertex_xy is None:
            X, Y = np.meshgrid(self.axis_nodes(self.vertex_x), self.axis_nodes(self.vertex_y))
            return X.ravel(), Y.ravel()
        P, xi = self.degree, gauss_lobatto(self.degree)
        I, J = np.meshgrid(np.arange(self.nfx), np.arange(self.nfy))
        cx, cy = np.minimum(I // P, self.n_cells_x - 1), np.minimum(J // P, self.n_cells_y - 1)
        s, t = xi[I - P * cx], xi[J - P * cy]
        v = self.vertex_xy
        out = []
        for k in range(2):
            out.append(((1 - s) * (1 - t) * v[cy, cx, k] + s * (1 - t) * v[cy, cx + 1, k]
                        + (1 - s) * t * v[cy + 1, cx, k] + s * t * v[cy + 1, cx + 1, k]).ravel())
        return out[0], out[1]

    def constrained(self):
        """Periodic images (deal.II's constrained DoFs): last column / row of a periodic direction."""
        c = np.zeros((self.nfy, self.nfx), bool)
        if self.periodic_x:
            c[:, -1] = True
        if self.periodic_y:
            c[-1, :] = True
        return c.ravel()

    def independent(self):
        return ~self.constrained()

    def master(self):
        """The source node of every structured node (itself unless a periodic image)."""
        I, J = np.meshgrid(np.arange(self.nfx), np.arange(self.nfy))
        if self.periodic_x:
            I = np.where(I == self.nfx - 1, 0, I)
        if self.periodic_y:
            J = np.where(J == self.nfy - 1, 0, J)
        return (J * self.nfx + I).ravel()

    def n_unique(self):
        return int(self.independent().sum())

    def time_step(self, cfl):
        """Discretization::time_step (discretization.h:158-162): cfl h_min / p^2."""
        return cfl * self.h_min / (self.degree * self.degree)


def build_mesh(tc: TestCase, n_cells_x: int, degree: int = 1, n_cells_y: int | None = None) -> Mesh:
    """The box [0, L]^2 with the periodicity, mesh transformation and walls of tc
    (discretization.h:78-144). n_cells_y defaults to n_cells_x; a rectangular
    mesh takes h_min = min(L/nx, L/ny) before the transformation."""
    ny = n_cells_x if n_cells_y is None else n_cells_y
    vx = np.linspace(0.0, tc.L, n_cells_x + 1)
    vy = np.linspace(0.0, tc.L, ny + 1)
    h_min = min(tc.L / n_cells_x, tc.L / ny)
    vx, vy, h_min = tc.transform_axes(vx, vy, h_min)
    m = Mesh(degree, n_cells_x, ny, tc.n_periodic >= 1, tc.n_periodic >= 2, np.asarray(vx, float),
             np.asarray(vy, float), h_min)
    if getattr(tc, "distort", 0.0):
        VX, VY = np.meshgrid(m.vertex_x, m.vertex_y)
        TX, TY = tc.transform_vertices(VX, VY)
        m.vertex_xy = np.stack([TX, TY], axis=-1)
    x, y = m.nodes()
    mask, ux, uy = tc.wall_velocity(x, y)
    m.wall_dof = np.nonzero(mask)[0].astype(np.int64)
    m.wall_velocity = np.stack([ux[mask], uy[mask]], axis=1).astype(np.float64)
    return m


def run_length(tc: TestCase, mesh: Mesh, cfl: float, t_end: float, max_steps: int = 0):
    """dt and the number of steps of the driver (cgdbe.cc:236-242)."""
    T = t_end * tc.reference_time()
    dt = mesh.time_step(cfl)
    n_steps = max_steps if max_steps > 0 else int(math.ceil(T / dt))
    if not tc.steady and max_steps == 0:
        dt = T / n_steps
    return dt, n_steps


def diagnostics(tc: TestCase, mesh: Mesh, weights: np.ndarray, f: np.ndarray, t: float, u_previous=None):
    """The nodal-quadrature monitors of cgdbe.cc:349-397 over the independent nodes:
    E/E0, exact E/E0, relative L2 velocity error, mean density drift, and the
    mean velocity change (|u - u_prev|, for the steady-state test)."""
    ind = mesh.independent()
    x, y = mesh.nodes()
    rho, ux, uy = d2q9.moments(f[:, ind])
    er, eux, euy = tc.exact(x[ind], y[ind], t)
    w = weights[ind]
    s0 = np.sum(w * ((ux - eux) ** 2 + (uy - euy) ** 2))
    s1 = np.sum(w * (eux ** 2 + euy ** 2))
    s2 = np.sum(w * (ux ** 2 + uy ** 2))
    s3 = np.sum(w * rho)
    s4 = np.sum(w)
    du = None
    if u_previous is not None:
        du = np.sum(w * np.hypot(ux - u_previous[0], uy - u_previous[1])) / s4
    E0 = tc.energy_scale()
    return {
        "E/E0": s2 / s4 / E0,
        "E/E0 exact": s1 / s4 / E0,
        "rel_l2_u": math.sqrt(s0 / max(s1, 1e-300)),
        "mass_drift": s3 / s4 - tc.rho0,
        "mean_du": du,
        "u": (ux, uy),
    }
