"""General quadrilaterals (the reference's --distort, test_cases.h:52-63, MappingQ1)
on the GPU through the C ABI, against the oracle, whose distortion runs reproduce
the reference's table (docs/results.md:222-233): every operator and whole runs
of both schemes with CG, lumped and iterated lumping, p = 1..3; the bar is the
FP64 one, relative L2 <= 1e-12 (operators, runs), <= 1e-14 (diagonals)."""
import numpy as np
import pytest

from helpers import directions, random_populations, rel_l2, setup_case, tgv
from lbfem_gpu import _abi, cases, d2q9, make_params

pytestmark = pytest.mark.gpu


def _gpu(mesh, params):
    import lbfem_gpu

    return lbfem_gpu.Solver(mesh, params)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_distorted_operators(gpu_lib, oracle_mod, p):
    tc, m = tgv(9, p=p, distort=0.05)
    g, o = _gpu(m, make_params()), oracle_mod.Oracle(m, make_params(cg_tolerance=1e-12))
    assert rel_l2(g.node_weight(), o.node_weight()) <= 1e-14
    assert rel_l2(g.jacobi_diagonal(), o.jacobi_diagonal()) <= 1e-14
    x = np.random.default_rng(p).standard_normal(m.n_dofs)
    assert rel_l2(g.mass_vmult(x), o.mass_vmult(x)) <= 1e-14
    f = random_populations(m, seed=p)
    feq = d2q9.equilibrium(*d2q9.moments(f))
    dt, lam = m.time_step(0.3), 2e-3
    for kind in ("taylor_galerkin", "leelin"):
        a = g.advection(f, directions(), dt, lam, kind=kind, feq=feq if kind == "leelin" else None)
        b = o.advection(f, directions(), dt, lam, kind=kind, feq=feq if kind == "leelin" else None)
        for al in range(8):
            assert rel_l2(a[al], b[al]) <= 1e-12, (kind, al, rel_l2(a[al], b[al]))
    g.close()
    g = _gpu(m, make_params(cg_tolerance=1e-12))
    r = x.copy()
    r[m.constrained()] = 0
    assert rel_l2(g.mass_solve(r), o.mass_solve(r)) <= 1e-12
    g.close()
    o.close()


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("scheme,mass", [("bardow", "cg"), ("leelin", "cg"), ("bardow", "lumped"),
                                         ("leelin", "richardson")])
def test_distorted_runs(gpu_lib, oracle_mod, p, scheme, mass):
    tc, m = tgv(8, p=p, distort=0.04)
    prm = make_params(scheme, mass, cg_tolerance=1e-12)
    dt, lam = m.time_step(0.25), tc.relaxation_time()
    out = []
    for backend in (_gpu, oracle_mod.Oracle):
        h = setup_case(backend, tc, m, prm, dt, lam)
        h.step(20)
        out.append(h.get_populations())
        h.close()
    assert rel_l2(out[0], out[1]) <= 1e-12


def test_distorted_error_table_on_the_gpu(gpu_lib):
    """The reference's 48^2 run at eps = 0.02 (docs/results.md:229): 1.81e-2."""
    tc, m = tgv(48, distort=0.02)
    dt, n = cases.run_length(tc, m, 0.25, 0.25)
    g = setup_case(_gpu, tc, m, make_params("bardow", "cg"), dt, tc.relaxation_time())
    g.step(n)
    err = cases.diagnostics(tc, m, g.node_weight(), g.get_populations(), n * dt)["rel_l2_u"]
    g.close()
    assert float(f"{err:.2e}") == 1.81e-2, err


def test_distorted_refusals(gpu_lib):
    tc, m = tgv(8, p=2, distort=0.04)
    for prm in (make_params(precision="mixed"), make_params(streaming="tg3")):
        with pytest.raises(_abi.LbfemError) as ei:
            _gpu(m, prm)
        assert ei.value.status == _abi.LBFEM_ERR_UNSUPPORTED
