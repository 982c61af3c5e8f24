"""The y-strip decomposition on the GPU: 2 and 3 strips of one mesh, each on
its own context of cuda:0, driven from one process (one host thread per
strip, LocalComm: the ghost rows and the sums move by device copies between
the strips' buffers on the host's word, so no kernel of one strip waits on
another's). FP64 strips against one whole-mesh context: relative L2 <= 1e-12
over the independent nodes (the strips sum dot products in another order).
Mixed-precision strips (whose window solves see the strip's own rows) against
the whole-mesh FP64 run: relative L2 velocity <= 1e-5."""
import numpy as np
import pytest

from helpers import rel_l2, setup_case
from lbfem_gpu import cases, d2q9, make_params, strips

pytestmark = pytest.mark.gpu


def _gpu(mesh, params):
    import lbfem_gpu

    return lbfem_gpu.Solver(mesh, params)


def _strip_run(tc, m, prm, dt, steps, n_ranks):
    lam = tc.relaxation_time()
    x, y = m.nodes()
    f0 = tc.initial_populations(x, y, lam)
    sol = strips.local_ranks(m, prm, n_ranks, _gpu, "cuda:0")
    strips.run_local(sol, lambda s: s.set_time_step(dt, lam))
    strips.run_local(sol, lambda s: s.set_initial_populations(f0))
    strips.run_local(sol, lambda s: s.step(steps))
    f = strips.assemble(m, [s.owned_populations() for s in sol])
    for s in sol:
        s.close()
    return f


def _case(name):
    if name == "tgv":
        tc = cases.TaylorGreenVortex(0.05, 1, 1)
        tc.set_reynolds(100)
        return tc, cases.build_mesh(tc, 16, 3), 0.5
    if name == "couette":
        tc = cases.CouetteFlow(0.1)
        tc.set_reynolds(10)
        return tc, cases.build_mesh(tc, 8, 1, n_cells_y=24), 0.25
    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(400)
    return tc, cases.build_mesh(tc, 16, 2), 0.4


@pytest.mark.parametrize("n_ranks", [2, 3])
@pytest.mark.parametrize("name,scheme,mass", [("tgv", "leelin", "cg"), ("cavity", "bardow", "cg"),
                                              ("cavity", "bardow", "lumped"), ("couette", "leelin", "cg"),
                                              ("tgv", "bardow", "richardson")])
def test_fp64_strips_match_one_context(gpu_lib, name, scheme, mass, n_ranks):
    tc, m, cfl = _case(name)
    prm = make_params(scheme, mass, cg_tolerance=1e-12)
    dt = m.time_step(cfl)
    h = setup_case(_gpu, tc, m, prm, dt, tc.relaxation_time())
    h.step(25)
    ref = h.get_populations()
    h.close()
    f = _strip_run(tc, m, prm, dt, 25, n_ranks)
    ind = m.independent()
    assert rel_l2(f[:, ind], ref[:, ind]) <= 1e-12


@pytest.mark.parametrize("name,scheme,mass", [("tgv", "leelin", "cg"), ("cavity", "bardow", "cg"),
                                              ("cavity", "bardow", "lumped")])
def test_mixed_strips_against_fp64(gpu_lib, name, scheme, mass):
    tc, m, cfl = _case(name)
    dt = m.time_step(cfl)
    h = setup_case(_gpu, tc, m, make_params(scheme, mass, cg_tolerance=1e-12), dt, tc.relaxation_time())
    h.step(100)
    ref = h.get_populations()
    h.close()
    f = _strip_run(tc, m, make_params(scheme, mass, precision="mixed"), dt, 100, 2)
    ind = m.independent()
    _, ux, uy = d2q9.moments(f[:, ind])
    _, rx, ry = d2q9.moments(ref[:, ind])
    assert rel_l2(np.stack([ux, uy]), np.stack([rx, ry])) <= 1e-5
