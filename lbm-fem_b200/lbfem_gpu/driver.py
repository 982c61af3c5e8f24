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


def reynolds_ladder(first, last, n):
    """n Reynolds numbers from first to last, geometrically spaced: the stages of a
    continuation (cgdbe's --Re list, cgdbe.cc:280-290)."""
    if n < 1:
        raise ValueError("a ladder has at least one rung")
    if n == 1:
        return [float(first)]
    return [first * (last / first) ** (k / (n - 1)) for k in range(n)]


def batched_ladder(solvers, steps_per_stage, *, batch=True):
    """A Reynolds-continuation ladder with its rungs as concurrent instances.

    cgdbe continues one Reynolds number after the other on the same populations:
    set_time_step with the next relaxation time, Scheme::f kept (cgdbe.cc:280-290).
    Here rung k is its own context, created with its own time step. Rung 0
    starts from the populations it holds. At stage k, rung k is warm-started from
    rung k - 1's populations at that moment (set_populations: the state only; the
    solver's start history restarts). Rungs 0..k then take steps_per_stage steps
    together, one graph launch per step of all of them (Batch) when batch is true,
    one rung after the other otherwise. The two give the same populations.
    Returns the steps each rung took."""
    from . import Batch

    n = len(solvers)
    taken = [0] * n
    for s in range(n):
        if s > 0:
            solvers[s].set_populations(solvers[s - 1].get_populations())
        active = solvers[: s + 1]
        if batch and len(active) > 1:
            b = Batch(active)
            try:
                b.step(steps_per_stage)
            finally:
                b.close()
        else:
            for h in active:
                h.step(steps_per_stage)
        for k in range(s + 1):
            taken[k] += steps_per_stage
    return taken
