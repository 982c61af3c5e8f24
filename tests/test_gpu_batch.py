"""Batched stepping of independent instances (lbfem_gpu_batch_step): every
instance ends where lbfem_gpu_step alone takes it, bitwise; a failing instance
is reported and left as before its failing step while the others finish."""
import math

import numpy as np
import pytest

from helpers import setup_case
from lbfem_gpu import cases, d2q9, make_params

pytestmark = pytest.mark.gpu


def _instances():
    """Uneven instances: cavities and Taylor-Green vortices, p = 1, 2, both schemes and precisions."""
    out = []
    table = [("cavity", 12, 2, "bardow", "fp64"), ("tgv", 16, 1, "leelin", "mixed"), ("cavity", 20, 1, "leelin", "fp64"),
             ("tgv", 10, 2, "bardow", "mixed"), ("cavity", 8, 2, "bardow", "mixed"), ("tgv", 24, 1, "bardow", "fp64")]
    for case, n, p, scheme, precision in table:
        if case == "tgv":
            tc = cases.TaylorGreenVortex(0.05 / math.sqrt(d2q9.CS2), 1, 1, shift=(0.25, 0.25), chapman_enskog=False)
            tc.set_reynolds(100)
        else:
            tc = cases.LidDrivenCavity(0.1, 1.2)
            tc.set_reynolds(400)
        m = cases.build_mesh(tc, n, p)
        out.append((tc, m, make_params(scheme, "cg", cg_tolerance=1e-10, precision=precision), m.time_step(0.4)))
    return out


def test_batch_matches_single_instances(gpu_lib):
    import lbfem_gpu

    batch_handles, single_handles = [], []
    for tc, m, prm, dt in _instances():
        batch_handles.append(setup_case(lbfem_gpu.Solver, tc, m, prm, dt, tc.relaxation_time()))
        single_handles.append(setup_case(lbfem_gpu.Solver, tc, m, prm, dt, tc.relaxation_time()))
    b = lbfem_gpu.Batch(batch_handles)
    b.step(5)
    b.step(4)  # a second call continues (the buffer states differ per instance)
    for h in single_handles:
        h.step(9)
    for hb, hs in zip(batch_handles, single_handles):
        assert np.array_equal(hb.get_populations(), hs.get_populations())
    b.close()


def test_batch_failure_of_one_instance(gpu_lib):
    import lbfem_gpu

    inst = _instances()[:3]
    handles = []
    for k, (tc, m, prm, dt) in enumerate(inst):
        if k == 1:  # an iteration cap of one in an FP64 solve at 1e-14: fails at its first step
            prm = make_params("bardow", "cg", cg_tolerance=1e-14, cg_max_iterations=1)
        handles.append(setup_case(lbfem_gpu.Solver, tc, m, prm, dt, tc.relaxation_time()))
    before = handles[1].get_populations()
    ref = setup_case(lbfem_gpu.Solver, inst[2][0], inst[2][1], inst[2][2], inst[2][3], inst[2][0].relaxation_time())
    ref.step(3)
    b = lbfem_gpu.Batch(handles)
    with pytest.raises(lbfem_gpu.NoConvergence) as ei:
        b.step(3)
    assert "instance 1" in str(ei.value)
    assert np.array_equal(handles[1].get_populations(), before)
    assert np.array_equal(handles[2].get_populations(), ref.get_populations())
    b.close()


def test_batch_with_tg3_instances(gpu_lib):
    """TG3 and split-TG3 instances (two solver loops per split step) in one batch
    with a TG2 instance: each ends where it ends alone, bitwise."""
    import lbfem_gpu

    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(400)
    table = [(12, 1, "tg3-split"), (8, 2, "tg3"), (10, 2, "tg2")]
    batch_handles, single_handles = [], []
    for n, p, streaming in table:
        m = cases.build_mesh(tc, n, p)
        prm = make_params("bardow", "cg", cg_tolerance=1e-10, streaming=streaming)
        dt = m.time_step(0.8)
        batch_handles.append(setup_case(lbfem_gpu.Solver, tc, m, prm, dt, tc.relaxation_time()))
        single_handles.append(setup_case(lbfem_gpu.Solver, tc, m, prm, dt, tc.relaxation_time()))
    b = lbfem_gpu.Batch(batch_handles)
    b.step(6)
    for h in single_handles:
        h.step(6)
    for hb, hs in zip(batch_handles, single_handles):
        assert np.array_equal(hb.get_populations(), hs.get_populations())
    b.close()


def _ladder(factory, precision, n_rungs, cells, p):
    """A continuation ladder of lid-driven cavities, Re 100 -> 400, rungs warm-started
    by driver.batched_ladder."""
    from lbfem_gpu import driver

    tc = cases.LidDrivenCavity(0.1, 1.2)
    m = cases.build_mesh(tc, cells, p)
    dt = m.time_step(0.4)
    x, y = m.nodes()
    hs = []
    for k, re in enumerate(driver.reynolds_ladder(100.0, 400.0, n_rungs)):
        tc.set_reynolds(re)
        h = factory(m, make_params("bardow", "cg", cg_tolerance=1e-12, precision=precision))
        h.set_time_step(dt, tc.relaxation_time())
        if k == 0:
            h.set_initial_populations(tc.initial_populations(x, y, tc.relaxation_time()))
        hs.append(h)
    return hs


def test_ladder_against_the_oracle(gpu_lib, oracle_mod):
    """The batched continuation ladder (one graph launch per step of the active
    rungs) against the same ladder on the FP64 oracle, rung by rung."""
    import lbfem_gpu
    from lbfem_gpu import driver

    g = _ladder(lbfem_gpu.Solver, "fp64", 3, 10, 1)
    o = _ladder(lambda m, prm: oracle_mod.Oracle(m, prm), "fp64", 3, 10, 1)
    assert driver.batched_ladder(g, 6, batch=True) == driver.batched_ladder(o, 6, batch=False) == [18, 12, 6]
    for a, b in zip(g, o):
        fa, fb = a.get_populations(), b.get_populations()
        assert np.linalg.norm(fa - fb) <= 1e-12 * np.linalg.norm(fb)


def test_ladder_batched_equals_one_at_a_time(gpu_lib):
    """Mixed precision, Q2: the batched ladder and the ladder stepped one rung at a
    time end bitwise equal."""
    import lbfem_gpu
    from lbfem_gpu import driver

    a = _ladder(lbfem_gpu.Solver, "mixed", 4, 8, 2)
    b = _ladder(lbfem_gpu.Solver, "mixed", 4, 8, 2)
    driver.batched_ladder(a, 5, batch=True)
    driver.batched_ladder(b, 5, batch=False)
    for x, y in zip(a, b):
        assert np.array_equal(x.get_populations(), y.get_populations())


def _grouped_instances():
    """Mixed-precision instances of every degree, both schemes and uneven sizes
    (the grouped launches), with two FP64 instances (graph branches beside them)."""
    out = []
    table = [("cavity", 24, 1, "bardow", "mixed"), ("tgv", 12, 2, "leelin", "mixed"), ("cavity", 6, 3, "bardow", "mixed"),
             ("tgv", 8, 4, "leelin", "mixed"), ("tgv", 30, 1, "leelin", "mixed"), ("cavity", 10, 2, "leelin", "mixed"),
             ("tgv", 6, 3, "bardow", "mixed"), ("cavity", 9, 1, "bardow", "fp64"), ("cavity", 5, 4, "bardow", "mixed"),
             ("tgv", 7, 2, "leelin", "fp64")]
    for k, (case, n, p, scheme, precision) in enumerate(table):
        if case == "tgv":
            tc = cases.TaylorGreenVortex((0.03 + 0.01 * k) / math.sqrt(d2q9.CS2), 1, 1, shift=(0.25, 0.25),
                                         chapman_enskog=False)
            tc.set_reynolds(100 + 50 * k)
        else:
            tc = cases.LidDrivenCavity(0.05 + 0.01 * k, 1.2)
            tc.set_reynolds(200 + 40 * k)
        m = cases.build_mesh(tc, n, p)
        # uneven tolerances: the instances' solves stop after different numbers of rounds
        tol = [1e-6, 1e-5, 1e-6, 1e-4][k % 4] if precision == "mixed" else 1e-10
        out.append((tc, m, make_params(scheme, "cg", cg_tolerance=tol, precision=precision), m.time_step(0.4)))
    return out


def _run(grouped, monkeypatch, n_first=4, n_second=3, host_driven=False):
    import lbfem_gpu

    monkeypatch.setenv("LBFEM_BATCH_GROUP", "1" if grouped else "0")
    hs = [setup_case(lbfem_gpu.Solver, tc, m, prm, dt, tc.relaxation_time()) for tc, m, prm, dt in _grouped_instances()]
    if host_driven:
        monkeypatch.setenv("LBFEM_TRACE", "1")  # read at batch creation: the grouped kernels one by one
    b = lbfem_gpu.Batch(hs)
    monkeypatch.delenv("LBFEM_TRACE", raising=False)
    b.step(n_first)
    # a new time step for two instances: the batch graph and its grouped tables are recorded again
    for k in (1, 7):
        tc, m, _, dt = _grouped_instances()[k]
        hs[k].set_time_step(0.9 * dt, tc.relaxation_time())
    b.step(n_second)
    launches = b.last_launches()
    b.close()
    return [h.get_populations() for h in hs], launches


def test_grouped_batch_matches_single_instances(gpu_lib, monkeypatch):
    """The grouped launches give every instance bitwise the populations of its own
    steps, and of the batch without grouping, with fewer kernel launches."""
    import lbfem_gpu

    singles = []
    for k, (tc, m, prm, dt) in enumerate(_grouped_instances()):
        h = setup_case(lbfem_gpu.Solver, tc, m, prm, dt, tc.relaxation_time())
        h.step(4)
        if k in (1, 7):
            h.set_time_step(0.9 * dt, tc.relaxation_time())
        h.step(3)
        singles.append(h.get_populations())
    grouped, n_grouped = _run(True, monkeypatch)
    branches, n_branches = _run(False, monkeypatch)
    host, n_host = _run(True, monkeypatch, host_driven=True)
    for k, (fg, fb, fh, fs) in enumerate(zip(grouped, branches, host, singles)):
        assert np.array_equal(fg, fs), k
        assert np.array_equal(fb, fs), k
        assert np.array_equal(fh, fs), k
    assert 0 < n_grouped < n_branches
    assert n_host == n_grouped


def test_grouped_batch_failure_of_one_instance(gpu_lib, monkeypatch):
    """A grouped instance whose solve stops at its round cap is reported and left as
    before its failing step; the other grouped instances complete all steps."""
    import lbfem_gpu

    monkeypatch.setenv("LBFEM_BATCH_GROUP", "1")
    inst = _grouped_instances()[:4]
    handles, refs = [], []
    for k, (tc, m, prm, dt) in enumerate(inst):
        if k == 2:  # a tolerance below the FP32 resolution: stagnates (or meets its cap) at its first step
            prm = make_params("bardow", "cg", cg_tolerance=1e-12, mixed_tolerance=1e-12, cg_max_iterations=4,
                              precision="mixed")
        handles.append(setup_case(lbfem_gpu.Solver, tc, m, prm, dt, tc.relaxation_time()))
        r = setup_case(lbfem_gpu.Solver, tc, m, prm, dt, tc.relaxation_time())
        if k != 2:
            r.step(3)
        refs.append(r)
    before = handles[2].get_populations()
    b = lbfem_gpu.Batch(handles)
    with pytest.raises(lbfem_gpu.NoConvergence) as ei:
        b.step(3)
    assert "instance 2" in str(ei.value)
    assert np.array_equal(handles[2].get_populations(), before)
    for k in (0, 1, 3):
        assert np.array_equal(handles[k].get_populations(), refs[k].get_populations()), k
    b.close()
