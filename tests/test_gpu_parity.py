"""Parity of the CUDA path (through the C ABI) with the CPU oracle on the same
seeded inputs: every operator of the hot path, then whole runs of both schemes.
FP64 bar: relative L2 <= 1e-12 (rounding order differs; CG stops on the same
tolerance), element-wise nodal maps <= 1e-14."""
import math

import numpy as np
import pytest

from helpers import directions, random_populations, rel_l2, setup_case, tgv, unit_mesh
from lbfem_gpu import _abi, cases, d2q9, make_params

pytestmark = pytest.mark.gpu


def _gpu(mesh, params, dof_index=None):
    import lbfem_gpu

    return lbfem_gpu.Solver(mesh, params, dof_index=dof_index)


def _meshes():
    out = []
    tc = cases.TaylorGreenVortex(0.05, 1, 4)
    tc.set_reynolds(100)
    out.append(("tgv", tc, 1, 12))
    tc = cases.CouetteFlow(0.1)
    tc.set_reynolds(10)
    out.append(("couette", tc, 1, 10))
    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(400)
    out.append(("cavity", tc, 1, 9))
    return out


MESHES = _meshes()


@pytest.mark.parametrize("name,tc,_p,n", MESHES, ids=[m[0] for m in MESHES])
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_nodal_maps(gpu_lib, oracle_mod, name, tc, _p, n, p):
    m = cases.build_mesh(tc, n, p)
    f = random_populations(m, seed=p)
    feq_in = random_populations(m, seed=p + 10)
    incr = 1e-3 * np.random.default_rng(p).standard_normal((8, m.n_dofs))
    g, o = _gpu(m, make_params()), oracle_mod.Oracle(m, make_params())
    for fn, args in (("collide_bgk", (f, 1.3)), ("compute_equilibrium", (f,)),
                     ("predictor_corrector", (f, feq_in, incr, 0.7))):
        a, b = getattr(g, fn)(*args), getattr(o, fn)(*args)
        assert np.max(np.abs(a - b)) <= 1e-14 * np.max(np.abs(b)), (fn, np.max(np.abs(a - b)))


@pytest.mark.parametrize("name,tc,_p,n", MESHES, ids=[m[0] for m in MESHES])
@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("kind", ["taylor_galerkin", "leelin"])
def test_advection(gpu_lib, oracle_mod, name, tc, _p, n, p, kind):
    m = cases.build_mesh(tc, n, p)
    f = random_populations(m, seed=3 * p)
    feq = d2q9.equilibrium(*d2q9.moments(f)) if kind == "leelin" else None
    dt, lam = m.time_step(0.3), 2e-3
    g, o = _gpu(m, make_params()), oracle_mod.Oracle(m, make_params())
    for rm in (-1, 0, 1):
        a = g.advection(f, directions(), dt, lam, kind=kind, feq=feq, remove_wall_mass_flux=rm)
        b = o.advection(f, directions(), dt, lam, kind=kind, feq=feq, remove_wall_mass_flux=rm)
        for al in range(8):
            assert rel_l2(a[al], b[al]) <= 1e-12, (al, rm, rel_l2(a[al], b[al]))
        assert np.all(a[:, m.constrained()] == 0)


@pytest.mark.parametrize("name,tc,_p,n", MESHES, ids=[m[0] for m in MESHES])
@pytest.mark.parametrize("p", [1, 2, 3])
def test_mass_operator(gpu_lib, oracle_mod, name, tc, _p, n, p):
    m = cases.build_mesh(tc, n, p)
    g, o = _gpu(m, make_params()), oracle_mod.Oracle(m, make_params())
    assert rel_l2(g.node_weight(), o.node_weight()) <= 1e-14
    assert rel_l2(g.jacobi_diagonal(), o.jacobi_diagonal()) <= 1e-14
    x = np.random.default_rng(7).standard_normal(m.n_dofs)
    assert rel_l2(g.mass_vmult(x), o.mass_vmult(x)) <= 1e-14


@pytest.mark.parametrize("name,tc,_p,n", MESHES, ids=[m[0] for m in MESHES])
@pytest.mark.parametrize("p", [1, 2])
@pytest.mark.parametrize("mass", ["cg", "lumped", "richardson"])
def test_mass_solve(gpu_lib, oracle_mod, name, tc, _p, n, p, mass):
    m = cases.build_mesh(tc, n, p)
    prm = make_params(mass=mass, cg_tolerance=1e-13)
    g, o = _gpu(m, prm), oracle_mod.Oracle(m, prm)
    rng = np.random.default_rng(11)
    r = rng.standard_normal(m.n_dofs)
    r[m.constrained()] = 0
    x0 = 0.1 * rng.standard_normal(m.n_dofs)
    x0[m.constrained()] = 0
    a, b = g.mass_solve(r, x=x0), o.mass_solve(r, x=x0)
    assert rel_l2(a, b) <= 1e-12
    assert abs(g.cg_iterations() - o.cg_iterations()) <= 1


def test_cg_no_convergence(gpu_lib):
    tc, m = tgv(8)
    g = _gpu(m, make_params(cg_tolerance=1e-14, cg_max_iterations=1))
    r = np.sin(np.arange(m.n_dofs) * 0.37)
    r[m.constrained()] = 0
    with pytest.raises(_abi.NoConvergence):
        g.mass_solve(r)


def test_state_and_argument_errors(gpu_lib):
    tc, m = tgv(8)
    g = _gpu(m, make_params())
    with pytest.raises(_abi.LbfemError) as ei:
        g.set_initial_populations(np.ones((9, m.n_dofs)))
    assert ei.value.status == _abi.LBFEM_ERR_STATE
    with pytest.raises(_abi.LbfemError) as ei:
        g.set_time_step(-1.0, 1.0)
    assert ei.value.status == _abi.LBFEM_ERR_ARG


def _run_pair(oracle_mod, tc, m, prm, dt, steps, lam=None):
    lam = tc.relaxation_time() if lam is None else lam
    g = setup_case(_gpu, tc, m, prm, dt, lam)
    o = setup_case(oracle_mod.Oracle, tc, m, prm, dt, lam)
    g.step(steps)
    o.step(steps)
    return g, o


@pytest.mark.parametrize("scheme,mass,case,p,n,steps", [
    ("bardow", "cg", "tgv", 1, 24, 60),
    ("leelin", "cg", "tgv", 2, 10, 40),
    ("bardow", "lumped", "cavity", 2, 8, 80),
    ("leelin", "cg", "couette", 1, 12, 80),
    ("bardow", "cg", "cavity", 1, 12, 60),
    ("leelin", "lumped", "cavity", 3, 5, 40),
    ("bardow", "cg", "couette", 3, 4, 40),
    ("bardow", "richardson", "cavity", 2, 10, 60),
    ("leelin", "richardson", "tgv", 1, 16, 50),
])
def test_step(gpu_lib, oracle_mod, scheme, mass, case, p, n, steps):
    if case == "tgv":
        tc = cases.TaylorGreenVortex(0.05, 1, 4)
        tc.set_reynolds(100)
    elif case == "couette":
        tc = cases.CouetteFlow(0.1)
        tc.set_reynolds(10)
    else:
        tc = cases.LidDrivenCavity(0.1, 1.2)
        tc.set_reynolds(400)
    m = cases.build_mesh(tc, n, p)
    prm = make_params(scheme, mass, cg_tolerance=1e-12)
    g, o = _run_pair(oracle_mod, tc, m, prm, m.time_step(0.3), steps)
    a, b = g.get_populations(), o.get_populations()
    assert rel_l2(a, b) <= 1e-12, rel_l2(a, b)
    if mass == "cg" and case != "couette":
        # Couette is uniform in x: the right-hand sides of the axis populations are pure round-off,
        # so their stopping iteration is noise; elsewhere the counts agree closely
        assert abs(g.cg_iterations() - o.cg_iterations()) <= 0.05 * o.cg_iterations() + 2
    ca, cb = g.conservation(), o.conservation()
    assert np.allclose(ca, cb, rtol=1e-12, atol=1e-15)


def test_tgv_plain_fp64_2000_steps(gpu_lib, oracle_mod):
    """Periodic TGV, 64 x 64 Q1, Bardow, consistent mass (Jacobi-PCG to 1e-12), Re 100,
    U0 = 0.05, CFL 0.5 on h, u = U0 sin(2 pi x) cos(2 pi y), f = feq, 2000 steps."""
    tc = cases.TaylorGreenVortex(0.05 / math.sqrt(d2q9.CS2), 1, 1, shift=(0.25, 0.25), chapman_enskog=False)
    tc.set_reynolds(100)
    m = cases.build_mesh(tc, 64, 1)
    prm = make_params("bardow", "cg", cg_tolerance=1e-12)
    g, o = _run_pair(oracle_mod, tc, m, prm, m.time_step(0.5), 2000)
    a, b = g.get_populations(), o.get_populations()
    err = rel_l2(a, b)
    assert err <= 1e-12, err
    ua = d2q9.moments(a[:, m.independent()])
    ub = d2q9.moments(b[:, m.independent()])
    assert rel_l2(np.stack(ua[1:]), np.stack(ub[1:])) <= 1e-12


def test_dof_permutation(gpu_lib):
    """A caller numbering (a permutation of the structured nodes) gives the same results."""
    tc, m = tgv(10, p=2)
    rng = np.random.default_rng(5)
    perm = rng.permutation(m.n_dofs).astype(np.int64)  # structured node s -> caller DoF perm[s]
    prm = make_params("bardow", "cg", cg_tolerance=1e-12)
    dt, lam = m.time_step(0.25), tc.relaxation_time()
    x, y = m.nodes()
    f0 = tc.initial_populations(x, y, lam)
    ref = _gpu(m, prm)
    ref.set_time_step(dt, lam)
    ref.set_initial_populations(f0)
    ref.step(20)
    # the same mesh with permuted numbering: walls would also be given by caller DoF
    g = _gpu(m, prm, dof_index=perm)
    fc = np.empty_like(f0)
    fc[:, perm] = f0
    g.set_time_step(dt, lam)
    g.set_initial_populations(fc)
    g.step(20)
    out = g.get_populations()
    assert np.array_equal(out[:, perm], ref.get_populations())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_failure_leaves_the_populations(gpu_lib, precision):
    """A solver failure inside graph-launched steps: step raises NoConvergence
    (the reference's SolverControl::NoConvergence out of Scheme::step), and the
    populations are those before the failing step."""
    tc = cases.TaylorGreenVortex(0.05 / math.sqrt(d2q9.CS2), 1, 1, shift=(0.25, 0.25), chapman_enskog=False)
    tc.set_reynolds(100)
    m = cases.build_mesh(tc, 16, 1)
    dt, lam = m.time_step(0.4), tc.relaxation_time()
    if precision == "fp64":
        prm = make_params("bardow", "cg", cg_tolerance=1e-14, cg_max_iterations=1)
    else:  # a tolerance below the FP32 resolution of the solution: the rounds stagnate
        prm = make_params("bardow", "cg", precision="mixed", mixed_tolerance=1e-12)
    g = setup_case(_gpu, tc, m, prm, dt, lam)
    before = g.get_populations()
    with pytest.raises(_abi.NoConvergence):
        g.step(3)
    assert np.array_equal(g.get_populations(), before)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_steps_match_host_driven_steps(gpu_lib, precision, monkeypatch):
    """The graph-launched steps (device-side solver loops) and the host-driven
    steps (LBFEM_TRACE) run the same kernels in the same order: bitwise equal."""
    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(400)
    m = cases.build_mesh(tc, 12, 2)
    dt, lam = m.time_step(0.4), tc.relaxation_time()
    prm = make_params("leelin", "cg", cg_tolerance=1e-10, precision=precision)
    g = setup_case(_gpu, tc, m, prm, dt, lam)
    monkeypatch.setenv("LBFEM_TRACE", "1")
    h = setup_case(_gpu, tc, m, prm, dt, lam)
    g.step(7)
    h.step(7)
    assert np.array_equal(g.get_populations(), h.get_populations())


@pytest.mark.parametrize("passes", [0, 1, 2, 3])
def test_richardson_passes(gpu_lib, oracle_mod, passes):
    """--mass richardson[k] (mass.h:193-202): k = 0 is the lumped solve; odd and even k
    end in the same buffer; each agrees with the oracle."""
    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(400)
    m = cases.build_mesh(tc, 8, 2)
    prm = make_params("bardow", "richardson", richardson=passes)
    g, o = _run_pair(oracle_mod, tc, m, prm, m.time_step(0.3), 30)
    assert rel_l2(g.get_populations(), o.get_populations()) <= 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_checkpoint_restart(gpu_lib, oracle_mod, tmp_path, precision):
    """write_checkpoint / read_checkpoint (io.h:137-165): a restarted context holds
    the same populations, and continues to the solver tolerance (the checkpoint,
    like the reference's, holds f only: the CG start history restarts). The file
    is the oracle's format."""
    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(400)
    m = cases.build_mesh(tc, 12, 2)
    dt, lam = m.time_step(0.4), tc.relaxation_time()
    prm = make_params("bardow", "cg", cg_tolerance=1e-12, precision=precision)
    a = setup_case(_gpu, tc, m, prm, dt, lam)
    a.step(10)
    name = str(tmp_path / "cavity")
    a.write_checkpoint(name)
    b = _gpu(m, prm)
    b.set_time_step(dt, lam)
    b.read_checkpoint(name)
    assert np.array_equal(b.get_populations(), a.get_populations())
    o = oracle_mod.Oracle(m, make_params("bardow", "cg", cg_tolerance=1e-12))
    o.read_checkpoint(name)
    assert np.array_equal(o.get_populations(), a.get_populations())
    a.step(10)
    b.step(10)
    assert rel_l2(b.get_populations(), a.get_populations()) <= (1e-10 if precision == "fp64" else 1e-6)


def test_cg_zero_rhs_nonzero_start_gives_zero(gpu_lib, oracle_mod):
    """As the oracle: an exactly zero right-hand side with a nonzero start
    returns x = 0 (deal.II's SolverCG would throw NoConvergence at the cap)."""
    tc, m = tgv(8)
    prm = make_params(cg_max_iterations=5)
    x0 = 1e-20 * np.cos(np.arange(m.n_dofs))
    for h in (_gpu(m, prm), oracle_mod.Oracle(m, prm)):
        x = h.mass_solve(np.zeros(m.n_dofs), x=x0)
        assert np.all(x == 0) and h.cg_iterations() == 0
        h.close()
