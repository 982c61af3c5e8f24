"""The y-strip decomposition (lbfem_gpu/strips.py) on CPU, with the oracle as
each rank's compute: the partition and its ghost rows, the exchanges and sums
the library makes through the strip callback, both communicators (threads in
one process, and world-size-2 gloo processes rendezvousing on 127.0.0.1), and
whole runs of both schemes against the single-rank oracle. The strips sum the
dot products in another order, so the bar is a relative L2 of 1e-12 over the
independent nodes (a periodic image row is not kept on strips)."""
import os
import socket
import sys

import numpy as np
import pytest

from helpers import rel_l2
from lbfem_gpu import cases, make_params, strips

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _oracle_run(oracle_mod, tc, m, prm, dt, steps):
    lam = tc.relaxation_time()
    x, y = m.nodes()
    h = oracle_mod.Oracle(m, prm)
    h.set_time_step(dt, lam)
    h.set_initial_populations(tc.initial_populations(x, y, lam))
    h.step(steps)
    f = h.get_populations()
    h.close()
    return f


def _strip_run(oracle_mod, tc, m, prm, dt, steps, n_ranks):
    lam = tc.relaxation_time()
    x, y = m.nodes()
    f0 = tc.initial_populations(x, y, lam)
    threads = oracle_mod.set_threads(0)
    oracle_mod.set_threads(1)  # one OpenMP thread per rank thread
    sol = strips.local_ranks(m, prm, n_ranks, lambda mm, pp: oracle_mod.Oracle(mm, pp), "cpu")
    strips.run_local(sol, lambda s: s.set_time_step(dt, lam))
    strips.run_local(sol, lambda s: s.set_initial_populations(f0))
    strips.run_local(sol, lambda s: s.step(steps))
    f = strips.assemble(m, [s.owned_populations() for s in sol])
    cons = sum(s.conservation_local() for s in sol)
    for s in sol:
        s.close()
    oracle_mod.set_threads(threads)
    return f, cons


def _cases():
    tgv = cases.TaylorGreenVortex(0.1, 1, 4)
    tgv.set_reynolds(100)
    cav = cases.LidDrivenCavity(0.1, 1.2)
    cav.set_reynolds(400)
    cou = cases.CouetteFlow(0.1)
    cou.set_reynolds(10)
    return {"tgv": (tgv, 12, None, 0.3), "cavity": (cav, 12, None, 0.4), "couette": (cou, 8, 16, 0.25)}


CASES = _cases()


def test_partition_rows_and_ghosts():
    tc, n, ny, _ = CASES["cavity"]
    m = cases.build_mesh(tc, n, 2, n_cells_y=ny)
    st = strips.partition(m, 3)
    own = np.concatenate([s.rows[s.own_rows] for s in st])
    assert np.array_equal(own, np.arange(m.nfy))  # every node row owned once, in order
    assert (st[0].below, st[0].ghost_below, st[-1].above, st[-1].ghost_above) == (None, 0, None, 0)
    for lo, hi in zip(st, st[1:]):
        # the upper strip's ghost rows below are the lower strip's last `degree` owned rows,
        # the lower strip's ghost row above is the upper strip's first owned row
        assert np.array_equal(hi.rows[:hi.ghost_below], lo.rows[lo.own_rows][-m.degree:])
        assert lo.rows[-1] == hi.rows[hi.own_rows][0]
    # periodic y: the first strip's ghosts wrap to the last one's rows, the last one's to row 0
    tc, n, _, _ = CASES["tgv"]
    m = cases.build_mesh(tc, n, 2)
    st = strips.partition(m, 2)
    assert list(st[0].rows[:2]) == [m.nfy - 3, m.nfy - 2] and st[-1].rows[-1] == 0
    with pytest.raises(ValueError):
        strips.partition(m, 7)  # fewer than 2 cell rows per strip


@pytest.mark.parametrize("n_ranks", [2, 3])
@pytest.mark.parametrize("name,scheme,mass", [("tgv", "leelin", "cg"), ("tgv", "bardow", "cg"),
                                              ("tgv", "bardow", "richardson"), ("cavity", "bardow", "cg"),
                                              ("cavity", "bardow", "lumped"), ("couette", "leelin", "cg")])
def test_strips_match_the_single_rank_oracle(oracle_mod, name, scheme, mass, n_ranks):
    tc, n, ny, cfl = CASES[name]
    p = 1 if name == "couette" else 2
    m = cases.build_mesh(tc, n, p, n_cells_y=ny)
    prm = make_params(scheme, mass, cg_tolerance=1e-12)
    dt = m.time_step(cfl)
    ref = _oracle_run(oracle_mod, tc, m, prm, dt, 10)
    f, cons = _strip_run(oracle_mod, tc, m, prm, dt, 10, n_ranks)
    ind = m.independent()
    assert rel_l2(f[:, ind], ref[:, ind]) <= 1e-12
    # the conservation sums over the owned rows add up to the single context's
    o = oracle_mod.Oracle(m, prm)
    o.set_populations(ref)
    assert np.allclose(cons, o.conservation(), rtol=1e-12, atol=1e-15)
    o.close()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      OMP_NUM_THREADS="2")
    for p in (ROOT, os.path.join(ROOT, "lbm-fem_b200"), os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    import oracle
    from lbfem_gpu import cases, make_params, strips

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    tc = cases.TaylorGreenVortex(0.1, 1, 4)
    tc.set_reynolds(100)
    m = cases.build_mesh(tc, 12, 2)
    lam, dt = tc.relaxation_time(), m.time_step(0.3)
    x, y = m.nodes()
    st = strips.partition(m, world)[rank]
    s = strips.StripSolver(m, st, make_params("leelin", "cg", cg_tolerance=1e-12),
                           lambda mm, pp: oracle.Oracle(mm, pp), "cpu",
                           lambda solver: strips.DistComm(st, solver.bufs))
    s.set_time_step(dt, lam)
    s.set_initial_populations(tc.initial_populations(x, y, lam))
    s.step(20)
    q.put((rank,) + s.owned_populations())
    s.close()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_strips_over_gloo_world_size_2(oracle_mod):
    """Two processes, one strip each, exchanging ghost rows and summing dot
    products over gloo (the path bench.py --gpus N takes with NCCL)."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    parts = sorted((q.get(timeout=240) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    tc, n, _, cfl = CASES["tgv"]
    m = cases.build_mesh(tc, n, 2)
    f = strips.assemble(m, [pt[1:] for pt in parts])
    ref = _oracle_run(oracle_mod, tc, m, make_params("leelin", "cg", cg_tolerance=1e-12), m.time_step(cfl), 20)
    ind = m.independent()
    assert rel_l2(f[:, ind], ref[:, ind]) <= 1e-12
