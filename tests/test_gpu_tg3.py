"""TG3 streaming on the GPU against the oracle: the streaming matrix
A = M + c K_e of MassSolver::solve (mass.h:57-129,185-213) for axis-parallel
and diagonal directions on periodic and walled meshes, whole TG3 and split-TG3
runs of the Bardow scheme (streaming.h:41-121), the reference's TG3 error
tables, and the failure / graph semantics of the two-sweep step. FP64 bar as
the other parity tests: relative L2 <= 1e-12."""
import numpy as np
import pytest

from helpers import rel_l2, setup_case, tgv
from lbfem_gpu import _abi, cases, make_params

pytestmark = pytest.mark.gpu


def _gpu(mesh, params):
    import lbfem_gpu

    return lbfem_gpu.Solver(mesh, params)


def _case(name):
    if name == "tgv":
        tc = cases.TaylorGreenVortex(0.05, 1, 4)
        tc.set_reynolds(100)
    elif name == "couette":
        tc = cases.CouetteFlow(0.1)
        tc.set_reynolds(10)
    else:
        tc = cases.LidDrivenCavity(0.1, 1.2)
        tc.set_reynolds(400)
    return tc


@pytest.mark.parametrize("name,n", [("tgv", 12), ("couette", 10), ("cavity", 9)])
@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("e", [(1.0, 0.0), (0.0, -1.0), (1.0, 1.0), (-1.0, 1.0)])
def test_tg3_mass_solve(gpu_lib, oracle_mod, name, n, p, e):
    tc = _case(name)
    m = cases.build_mesh(tc, n, p)
    prm = make_params("bardow", "cg", cg_tolerance=1e-13, streaming="tg3")
    g, o = _gpu(m, prm), oracle_mod.Oracle(m, prm)
    rng = np.random.default_rng(5 * p + n)
    r = rng.standard_normal(m.n_dofs)
    r[m.constrained()] = 0
    x0 = 0.1 * rng.standard_normal(m.n_dofs)
    x0[m.constrained()] = 0
    dt = m.time_step(1.0)
    c = dt * dt / 6
    a = g.mass_solve(r, x=x0, e=e, tg3_coefficient=c)
    b = o.mass_solve(r, x=x0, e=e, tg3_coefficient=c)
    assert rel_l2(a, b) <= 1e-12, rel_l2(a, b)
    assert abs(g.cg_iterations() - o.cg_iterations()) <= 1


@pytest.mark.parametrize("streaming,case,p,n,steps,cfl", [
    ("tg3", "tgv", 1, 24, 31, 1.0),
    ("tg3-split", "tgv", 1, 24, 31, 1.0),
    ("tg3", "tgv", 2, 10, 20, 0.5),
    ("tg3-split", "tgv", 3, 6, 20, 1.0),
    ("tg3", "cavity", 2, 8, 30, 0.6),
    ("tg3-split", "cavity", 1, 12, 40, 1.0),
    ("tg3-split", "couette", 2, 6, 30, 1.0),
])
def test_tg3_step(gpu_lib, oracle_mod, streaming, case, p, n, steps, cfl):
    tc = _case(case)
    m = cases.build_mesh(tc, n, p)
    prm = make_params("bardow", "cg", cg_tolerance=1e-12, streaming=streaming)
    dt, lam = m.time_step(cfl), tc.relaxation_time()
    g = setup_case(_gpu, tc, m, prm, dt, lam)
    o = setup_case(oracle_mod.Oracle, tc, m, prm, dt, lam)
    g.step(steps)
    o.step(steps)
    a, b = g.get_populations(), o.get_populations()
    assert rel_l2(a, b) <= 1e-12, rel_l2(a, b)
    if case != "couette":
        assert abs(g.cg_iterations() - o.cg_iterations()) <= 0.05 * o.cg_iterations() + 2
    assert np.allclose(g.conservation(), o.conservation(), rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("N,streaming,expected,its", [
    (24, "tg3", 1.04e-1, 5.1),
    (32, "tg3-split", 2.15e-2, None),
])
def test_tg3_error_table(gpu_lib, N, streaming, expected, its):
    """docs/results.md:97-107 and :143-149 (bardow, consistent mass, modes (1,4),
    Re 100, CFL 1, t = t_ref/4, Ma 0.05), to the printed digits, on the GPU."""
    tc, m = tgv(N)
    dt, n = cases.run_length(tc, m, 1.0, 0.25)
    g = setup_case(_gpu, tc, m, make_params("bardow", "cg", streaming=streaming), dt, tc.relaxation_time())
    g.step(n)
    err = cases.diagnostics(tc, m, g.node_weight(), g.get_populations(), n * dt)["rel_l2_u"]
    assert float(f"{err:.2e}") == expected, err
    if its is not None:
        assert round(g.cg_iterations() / (8 * n), 1) == its


@pytest.mark.parametrize("streaming", ["tg3", "tg3-split"])
def test_tg3_graph_steps_match_host_driven_steps(gpu_lib, streaming, monkeypatch):
    """Graph-launched TG3 steps (two WHILE loops per split step) and host-driven
    ones run the same kernels in the same order: bitwise equal."""
    tc = _case("cavity")
    m = cases.build_mesh(tc, 12, 2)
    dt, lam = m.time_step(0.8), tc.relaxation_time()
    prm = make_params("bardow", "cg", cg_tolerance=1e-10, streaming=streaming)
    g = setup_case(_gpu, tc, m, prm, dt, lam)
    monkeypatch.setenv("LBFEM_TRACE", "1")
    h = setup_case(_gpu, tc, m, prm, dt, lam)
    g.step(7)
    h.step(7)
    assert np.array_equal(g.get_populations(), h.get_populations())


@pytest.mark.parametrize("streaming", ["tg3", "tg3-split"])
def test_tg3_step_failure_leaves_the_populations(gpu_lib, streaming):
    """A CG failure in either sweep: NoConvergence, and the populations are
    those before the failing step (the first sweep's update went to the other
    population buffer)."""
    tc = _case("tgv")
    m = cases.build_mesh(tc, 16, 1)
    dt, lam = m.time_step(1.0), tc.relaxation_time()
    ok = make_params("bardow", "cg", cg_tolerance=1e-8, streaming=streaming)
    g = setup_case(_gpu, tc, m, ok, dt, lam)
    g.step(2)
    before = g.get_populations()
    bad = make_params("bardow", "cg", cg_tolerance=1e-14, cg_max_iterations=1, streaming=streaming)
    h = _gpu(m, bad)
    h.set_time_step(dt, lam)
    h.set_populations(before)
    with pytest.raises(_abi.NoConvergence):
        h.step(3)
    assert np.array_equal(h.get_populations(), before)


def test_tg3_settings_rejected(gpu_lib):
    """TG3 needs Bardow and the consistent mass (streaming.h:51-52, schemes.h:87);
    the mixed-precision path streams with TG2 only."""
    tc, m = tgv(8)
    for scheme, mass in (("leelin", "cg"), ("bardow", "lumped"), ("bardow", "richardson")):
        with pytest.raises(_abi.LbfemError) as ei:
            _gpu(m, make_params(scheme, mass, streaming="tg3"))
        assert ei.value.status == _abi.LBFEM_ERR_ARG
    with pytest.raises(_abi.LbfemError) as ei:
        _gpu(m, make_params("bardow", "cg", streaming="tg3-split", precision="mixed"))
    assert ei.value.status == _abi.LBFEM_ERR_UNSUPPORTED


@pytest.mark.parametrize("N,streaming,cfl,expected", [
    (64, "tg2", 0.25, 7.58e-3),
    (96, "tg2", 0.25, 2.89e-3),
    (64, "tg3", 1.0, 6.76e-3),
    (96, "tg3", 1.0, 2.84e-3),
    (64, "tg3-split", 1.0, 3.56e-3),
    (96, "tg3-split", 1.0, 2.16e-3),
])
def test_error_tables_at_larger_meshes(gpu_lib, N, streaming, cfl, expected):
    """docs/results.md:97-107,143-149 at N = 64 and 96 (bardow, consistent mass,
    modes (1,4), Re 100, t = t_ref/4, Ma 0.05), to the printed digits: the sizes
    the CPU oracle tests leave out."""
    tc, m = tgv(N)
    dt, n = cases.run_length(tc, m, cfl, 0.25)
    g = setup_case(_gpu, tc, m, make_params("bardow", "cg", streaming=streaming), dt, tc.relaxation_time())
    g.step(n)
    err = cases.diagnostics(tc, m, g.node_weight(), g.get_populations(), n * dt)["rel_l2_u"]
    assert float(f"{err:.2e}") == expected, err
