"""The gnuplot field files of the reference driver (cgdbe.cc:399-472, io.h:98-135).

``write_gnuplot`` writes the nodal rows of a context's populations as the
reference does: Taylor-Green and Couette ``x y u/U0 v/U0 |u|/U0``; the steady
cavity ``x y u/U0 v/U0 psi/(U0 L) rho-rho0`` with the stream function solved
on the device (``lbfem_gpu_stream_function``) and the vortex extrema of Ghia,
Ghia & Shin's Table I. Rows are sorted by y, then x, with a blank line between
grid rows (gnuplot's splot format); numbers are printed as C++ streams print a
double by default (``%g``).
"""
from __future__ import annotations

import numpy as np

from . import d2q9


def _g(v):
    return f"{float(v):g}"


def nodal_rows(handle, mesh, tc, steady):
    """The rows of every stored node (cgdbe.cc:405-446): moments of the
    populations (the periodic images take their source's populations first, as
    constraints.distribute does), the wall velocity on the wall nodes, and for a
    steady case the stream function psi / L in column 4."""
    f = handle.get_populations()[:, mesh.master()]
    rho, ux, uy = d2q9.moments(f)
    x, y = mesh.nodes()
    u, v = ux / tc.U0, uy / tc.U0
    if len(mesh.wall_dof):
        u[mesh.wall_dof] = mesh.wall_velocity[:, 0] / tc.U0
        v[mesh.wall_dof] = mesh.wall_velocity[:, 1] / tc.U0
    col4 = np.hypot(u, v)
    if steady:
        col4 = handle.stream_function(np.stack([u, v])) / tc.L
    return np.stack([x, y, u, v, col4, rho - tc.rho0], axis=1)


def sort_rows(rows, L):
    """write_grid_rows (io.h:98-135): by y (rounded to 2^-40 L), then x; returns the
    sorted rows and the index of the first row of each grid row."""
    key = np.rint(rows[:, 1] / L * float(1 << 40)).astype(np.int64)
    order = np.lexsort((rows[:, 0], key))
    key = key[order]
    starts = np.flatnonzero(np.r_[True, key[1:] != key[:-1]])
    return rows[order], starts


def vortex_extrema(rows):
    """The stream function extrema of cgdbe.cc:452-471 (label, psi, x, y): the
    primary vortex (max psi), and the minima in the lower left and lower right
    quarters of the unit cavity; the first row wins a tie, as in the reference."""
    out = []
    for label, sign, inside in (("primary vortex", 1.0, np.ones(len(rows), bool)),
                                ("lower left vortex", -1.0, (rows[:, 0] < 0.5) & (rows[:, 1] < 0.5)),
                                ("lower right vortex", -1.0, (rows[:, 0] > 0.5) & (rows[:, 1] < 0.5))):
        idx = np.flatnonzero(inside)
        best = idx[np.argmax(sign * rows[idx, 4])]
        out.append((label, rows[best, 4], rows[best, 0], rows[best, 1]))
    return out


def gnuplot_text(handle, mesh, tc, *, t_over_tref, step, reynolds, mach, n_cells, steady=None):
    """The text of the reference's gnuplot file of the current state."""
    steady = bool(getattr(tc, "steady", False)) if steady is None else steady
    rows, starts = sort_rows(nodal_rows(handle, mesh, tc, steady), tc.L)
    ncol = 6 if steady else 5
    lines = [f"# t/t_ref = {_g(t_over_tref)} (step {int(step)}), Re = {_g(reynolds)}, Ma = {_g(mach)}, "
             f"{int(n_cells)}^2 Q{mesh.degree} elements\n",
             "# x y u/U0 v/U0 psi/(U0 L) rho-rho0\n" if steady else "# x y u/U0 v/U0 |u|/U0\n"]
    first = set(starts[1:].tolist())
    for i, r in enumerate(rows):
        if i in first:
            lines.append("\n")
        lines.append("".join(_g(r[c]) + " " for c in range(ncol)) + "\n")
    if steady:
        for label, psi, x, y in vortex_extrema(rows):
            lines.append(f"# {label}: psi = {_g(psi)} at {_g(x)} {_g(y)}\n")
    return "".join(lines)


def write_gnuplot(path, handle, mesh, tc, **kw):
    """Writes gnuplot_text(...) to path (cgdbe.cc:399-472)."""
    with open(path, "w") as fh:
        fh.write(gnuplot_text(handle, mesh, tc, **kw))
