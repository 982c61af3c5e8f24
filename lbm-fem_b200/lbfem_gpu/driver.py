"""The time loop of the reference driver for steady cases (cgdbe.cc:270-397).

``steady_state`` runs one Reynolds number of a steady case on a context the way
``cgdbe`` does: steps in intervals of one reference time, the nodal-quadrature
monitor of the mean velocity change per reference time after each interval,
and a stop when it falls below the tolerance (``--steady-tol``, default 1e-4)
or at ``t_end`` reference times (default 100 for the cavity). A list of
Reynolds numbers is a continuation: call it again after ``set_time_step`` with
the next number's relaxation time, from the populations it left.
"""
from __future__ import annotations

import math

from .cases import diagnostics


def steady_state(handle, mesh, tc, dt, *, steady_tol=1e-4, t_end=100.0):
    """Returns (steps, converged, rate): the steps taken, whether the mean
    velocity change per reference time fell below steady_tol, and its last value."""
    t_ref = tc.reference_time()
    n_max = int(math.ceil(t_end * t_ref / dt))
    interval = max(1, int(round(t_ref / dt)))
    w = handle.node_weight()
    u_prev = diagnostics(tc, mesh, w, handle.get_populations(), 0.0)["u"]
    steps, t_prev, rate = 0, 0.0, 1.0
    while steps < n_max:
        n = min(interval, n_max - steps)
        handle.step(n)
        steps += n
        t = steps * dt
        d = diagnostics(tc, mesh, w, handle.get_populations(), t, u_prev)
        rate = d["mean_du"] / tc.U0 / ((t - t_prev) / t_ref)
        u_prev, t_prev = d["u"], t
        if rate < steady_tol:
            return steps, True, rate
    return steps, False, rate
