"""Parity at the sizes the benchmark configurations specify, through the C ABI:

* the start-up Couette flow on 32 x 256 Q1 cells (periodic in x), Lee-Lin,
  CFL 0.25, Re 50, top wall at U = 0.05, fluid at rest, 5000 steps: the FP64
  GPU path against the oracle (relative L2 of the populations <= 1e-12), the
  mixed path against the FP64 path (relative L2 velocity <= 1e-5), and both
  against the analytic series solution (test_cases.h:209-264);
* the lid-driven cavity on 128 x 128 Q2 cells (66049 nodes), Bardow, lumped
  and consistent mass, lid 0.1, Re 400, stretch 1.2, CFL 0.4: FP64 against the
  oracle and mixed against FP64 after a few thousand steps.

CG tolerance of the FP64 runs: 1e-12, the plain method's (config 0), so that
the FP64 comparison measures rounding, not where two CG runs of tolerance 1e-8
happen to stop (at 1e-8 the Couette run ends 7.4e-12 apart after 5000 steps).
The mixed runs use their own tolerance (LBFEM_MIXED_TOLERANCE). Mixed bar: 1e-5."""

TOL = 1e-12
import math

import numpy as np
import pytest

from helpers import rel_l2, setup_case
from lbfem_gpu import cases, d2q9, make_params

pytestmark = pytest.mark.gpu


def _gpu(mesh, params):
    import lbfem_gpu

    return lbfem_gpu.Solver(mesh, params)


def _run(backend, tc, mesh, params, dt, steps):
    h = setup_case(backend, tc, mesh, params, dt, tc.relaxation_time())
    h.step(steps)
    f = h.get_populations()
    w = h.node_weight()
    h.close()
    return f, w


def _velocity(mesh, f):
    _, ux, uy = d2q9.moments(f[:, mesh.independent()])
    return np.stack([ux, uy])


def test_config1_couette_32x256_5000_steps(gpu_lib, oracle_mod):
    tc = cases.CouetteFlow(0.05 / math.sqrt(d2q9.CS2))
    tc.set_reynolds(50)
    m = cases.build_mesh(tc, 32, 1, n_cells_y=256)
    dt, steps = m.time_step(0.25), 5000
    f_or, w = _run(oracle_mod.Oracle, tc, m, make_params("leelin", "cg", cg_tolerance=TOL), dt, steps)
    f64, _ = _run(_gpu, tc, m, make_params("leelin", "cg", cg_tolerance=TOL), dt, steps)
    fmx, _ = _run(_gpu, tc, m, make_params("leelin", "cg", precision="mixed"), dt, steps)
    assert rel_l2(f64, f_or) <= 1e-12, rel_l2(f64, f_or)
    e_u = rel_l2(_velocity(m, fmx), _velocity(m, f64))
    assert e_u <= 1e-5, e_u
    # the velocity profile against the analytic start-up solution, at t = 5000 dt
    t = steps * dt
    d_or = cases.diagnostics(tc, m, w, f_or, t)
    d64 = cases.diagnostics(tc, m, w, f64, t)
    dmx = cases.diagnostics(tc, m, w, fmx, t)
    assert abs(d64["rel_l2_u"] - d_or["rel_l2_u"]) <= 1e-9 * d_or["rel_l2_u"]
    assert d64["rel_l2_u"] < 1e-3, d64["rel_l2_u"]  # 3.35e-4 on this mesh
    assert abs(dmx["rel_l2_u"] - d64["rel_l2_u"]) <= 0.01 * d64["rel_l2_u"]
    assert abs(dmx["mass_drift"]) <= 1e-7


@pytest.mark.parametrize("mass,steps", [("lumped", 3000), ("cg", 1000)])
def test_config2_cavity_128_q2(gpu_lib, oracle_mod, mass, steps):
    tc = cases.LidDrivenCavity(0.1 / math.sqrt(d2q9.CS2), 1.2)
    tc.set_reynolds(400)
    m = cases.build_mesh(tc, 128, 2)
    assert m.n_dofs == 66049
    dt = m.time_step(0.4)
    f_or, _ = _run(oracle_mod.Oracle, tc, m, make_params("bardow", mass, cg_tolerance=TOL), dt, steps)
    f64, _ = _run(_gpu, tc, m, make_params("bardow", mass, cg_tolerance=TOL), dt, steps)
    fmx, _ = _run(_gpu, tc, m, make_params("bardow", mass, precision="mixed"), dt, steps)
    assert rel_l2(f64, f_or) <= 1e-12, rel_l2(f64, f_or)
    e_u = rel_l2(_velocity(m, fmx), _velocity(m, f64))
    assert e_u <= 1e-5, e_u
