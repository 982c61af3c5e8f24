"""The stream function (compute_stream_function, io.h:31-95) and the gnuplot
writer (cgdbe.cc:399-472) through the CUDA library, against the oracle and the
reference's own steady cavity result."""
import gzip
import os

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import rel_l2
from lbfem_gpu import cases, d2q9, make_params

pytestmark = pytest.mark.gpu


def _gpu(mesh, params):
    import lbfem_gpu

    return lbfem_gpu.Solver(mesh, params)


def _cavity_golden():
    text = gzip.open(os.path.join(GOLDEN, "cavity_Re1000.dat.gz"), "rt").read()
    rows = np.array([ln.split() for ln in text.splitlines() if ln.strip() and not ln.startswith("#")], float)
    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(1000)
    return text, rows, tc, cases.build_mesh(tc, 32, 2)


def test_stream_function_of_the_reference_cavity(gpu_lib, oracle_mod):
    text, rows, tc, m = _cavity_golden()
    vel = np.stack([rows[:, 2], rows[:, 3]])
    prm = make_params("bardow", "lumped")
    a = _gpu(m, prm).stream_function(vel)
    b = oracle_mod.Oracle(m, prm).stream_function(vel)
    assert rel_l2(a, b) <= 1e-10, rel_l2(a, b)
    assert np.max(np.abs(a / tc.L - rows[:, 4])) < 1e-6


@pytest.mark.parametrize("name", ["cavity", "tgv", "couette"])
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_stream_function(gpu_lib, oracle_mod, name, p):
    if name == "cavity":
        tc = cases.LidDrivenCavity(0.1, 1.2)
    elif name == "tgv":
        tc = cases.TaylorGreenVortex(0.05, 1, 4)
    else:
        tc = cases.CouetteFlow(0.1)
    tc.set_reynolds(100)
    m = cases.build_mesh(tc, 9, p)
    x, y = m.nodes()
    rng = np.random.default_rng(p)
    u = np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) + 0.1 * rng.standard_normal(x.shape)
    v = -np.cos(2 * np.pi * x) * np.sin(2 * np.pi * y) + 0.1 * rng.standard_normal(x.shape)
    vel = np.stack([u, v])[:, m.master()]  # periodic images carry their source's value
    prm = make_params("bardow", "cg")
    a = _gpu(m, prm).stream_function(vel)
    b = oracle_mod.Oracle(m, prm).stream_function(vel)
    assert rel_l2(a, b) <= 1e-10, rel_l2(a, b)


def test_gnuplot_writer_through_the_gpu(gpu_lib, oracle_mod):
    from lbfem_gpu import io

    text, rows, tc, m = _cavity_golden()
    f = d2q9.equilibrium(1 + rows[:, 5], rows[:, 2] * tc.U0, rows[:, 3] * tc.U0)
    outs = []
    for h in (_gpu(m, make_params("bardow", "lumped")), oracle_mod.Oracle(m, make_params("bardow", "lumped"))):
        h.set_time_step(1e-3, 1e-3)
        h.set_populations(f)
        outs.append(io.gnuplot_text(h, m, tc, t_over_tref=32.9998, step=391314, reynolds=1000, mach=0.1,
                                    n_cells=32))
    a, b = outs[0].splitlines(), outs[1].splitlines()
    assert len(a) == len(b) == len(text.splitlines())
    diff = [(la, lb) for la, lb in zip(a, b) if la != lb]
    assert len(diff) <= 0.01 * len(a), diff[:5]


def test_cavity_continuation_against_ghia(gpu_lib, oracle_mod):
    """The reference's CI run (ci.yml:44-58: cavity 16^2 Q1, Bardow, lumped, CFL 0.4,
    Re 100 then 400) on the GPU: the same steady states as the oracle (same step
    counts, psi within 1e-9) and psi_max within 10% of Ghia, Ghia & Shin."""
    from helpers import setup_case
    from lbfem_gpu import driver, io

    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(100)
    m = cases.build_mesh(tc, 16, 1)
    dt = m.time_step(0.4)
    prm = make_params("bardow", "lumped")
    g = setup_case(_gpu, tc, m, prm, dt, tc.relaxation_time())
    o = setup_case(oracle_mod.Oracle, tc, m, prm, dt, tc.relaxation_time())
    for Re, ghia in ((100, 0.1034), (400, 0.1139)):
        if Re != 100:
            tc.set_reynolds(Re)
            g.set_time_step(dt, tc.relaxation_time())
            o.set_time_step(dt, tc.relaxation_time())
        sg, cg, _ = driver.steady_state(g, m, tc, dt)
        so, co, _ = driver.steady_state(o, m, tc, dt)
        assert cg and co and sg == so
        psi = [io.nodal_rows(h, m, tc, True)[:, 4] for h in (g, o)]
        assert rel_l2(psi[0], psi[1]) <= 1e-9, rel_l2(psi[0], psi[1])
        assert abs(psi[0].max() - ghia) <= 0.1 * ghia, (Re, psi[0].max())
