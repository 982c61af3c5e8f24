"""The CPU oracle pinned against the reference: its compile-time lattice
identities, the element stencils of analysis/stencils.py, the amplification
factors of analysis/tg_spectral.py, the check value of
benchmarks/stencil_bench.cc, and the accuracy tables of docs/results.md."""
import json
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN
from helpers import directions, rel_l2, setup_case, tgv, unit_mesh
from lbfem_gpu import _abi, cases, d2q9, make_params
from lbfem_gpu._abi import LbfemError


# ------------------------------------------------------------- lattice KATs
def test_lattice_isotropy():
    """d2q9.h:80-88: sum_a w_a e..e = 1, 0, cs2 delta, 0, cs4 (delta delta + ...)."""
    cs2 = d2q9.CS2
    assert abs(d2q9.lattice_tensor() - 1) < 1e-14
    for i in (0, 1):
        assert abs(d2q9.lattice_tensor(i)) < 1e-14
    assert abs(d2q9.lattice_tensor(0, 0) - cs2) < 1e-14 and abs(d2q9.lattice_tensor(1, 1) - cs2) < 1e-14
    assert abs(d2q9.lattice_tensor(0, 1)) < 1e-14
    assert abs(d2q9.lattice_tensor(0, 0, 0)) < 1e-14 and abs(d2q9.lattice_tensor(0, 1, 1)) < 1e-14
    assert abs(d2q9.lattice_tensor(0, 0, 0, 0) - 3 * cs2 * cs2) < 1e-14
    assert abs(d2q9.lattice_tensor(0, 0, 1, 1) - cs2 * cs2) < 1e-14
    assert abs(d2q9.lattice_tensor(0, 0, 0, 1)) < 1e-14


def test_equilibrium_roundtrip_oracle(oracle_mod):
    """d2q9.h:89-92: moments(equilibrium(1.1, 0.05, -0.02)) round trip, through the oracle's nodal map."""
    m = unit_mesh(2, 1)
    o = oracle_mod.Oracle(m, make_params())
    f = np.tile(d2q9.equilibrium(1.1, 0.05, -0.02)[:, None], (1, m.n_dofs))
    feq = o.compute_equilibrium(f)
    rho, ux, uy = d2q9.moments(feq)
    assert np.all(np.abs(rho - 1.1) < 1e-14)
    assert np.all(np.abs(ux - 0.05) < 1e-14) and np.all(np.abs(uy + 0.02) < 1e-14)


# ----------------------------------------------------------- stencil KATs
def _stencil_rows(o, m, node, dt_pair=(1.0, 2.0)):
    """Rows of M, C_e, K_e at `node` for e = e_1..e_4, by applying the oracle to unit vectors."""
    p = m.degree
    e = directions()
    out = {"M": {}, "C": {a: {} for a in range(4)}, "K": {a: {} for a in range(4)}}
    i0, j0 = node
    for dy in range(-p, p + 1):
        for dx in range(-p, p + 1):
            u = np.zeros(m.n_dofs)
            u[(j0 + dy) * m.nfx + (i0 + dx)] = 1.0
            Mu = o.mass_vmult(u)
            out["M"][(dx, dy)] = Mu[j0 * m.nfx + i0]
            f = np.tile(u, (9, 1))
            r1 = o.advection(f, e, dt_pair[0], 1.0)
            r2 = o.advection(f, e, dt_pair[1], 1.0)
            for a in range(4):
                a1, a2 = r1[a, j0 * m.nfx + i0], r2[a, j0 * m.nfx + i0]
                K = 2 * a1 - a2  # r(dt) = -dt C u - dt^2/2 K u
                out["K"][a][(dx, dy)] = K
                out["C"][a][(dx, dy)] = -a1 - K / 2
    return out


@pytest.mark.parametrize("p", [1, 2])
def test_element_stencils(oracle_mod, p):
    """Assembled M, C_e, K_e stencils equal the reference's sympy stencils (analysis/stencils.py)."""
    gold = json.load(open(os.path.join(GOLDEN, "stencils.json")))
    m = unit_mesh(6, p)  # cell size 1: the stencils at h = 1
    o = oracle_mod.Oracle(m, make_params())
    names = {0: "(1,0)", 1: "(1,1)", 2: "(0,1)", 3: "(-1,1)"}
    for tx in range(p):
        for ty in range(p):
            rows = _stencil_rows(o, m, (2 * p + tx, 2 * p + ty))
            g = gold[f"Q{p} M"][f"{tx},{ty}"]
            for (dx, dy), v in rows["M"].items():
                assert abs(v - g.get(f"{dx},{dy}", 0.0)) < 1e-13, ("M", tx, ty, dx, dy)
            for a, en in names.items():
                for lab in ("C", "K"):
                    g = gold[f"Q{p} {lab} e={en}"][f"{tx},{ty}"]
                    for (dx, dy), v in rows[lab][a].items():
                        assert abs(v - g.get(f"{dx},{dy}", 0.0)) < 1e-12, (lab, en, tx, ty, dx, dy, v)


def test_amplification_factor(oracle_mod):
    """One TG2 or TG3 streaming step of a Fourier mode (consistent mass; TG3 with
    A = M + dt^2/6 K_e on the left) equals G_2d of analysis/tg_spectral.py."""
    gold = json.load(open(os.path.join(GOLDEN, "tg_spectral.json")))["cases"]
    n = 16
    m = unit_mesh(n, 1)
    o = oracle_mod.Oracle(m, make_params(cg_tolerance=1e-14, cg_max_iterations=500))
    e = directions()
    I, J = np.meshgrid(np.arange(m.nfx), np.arange(m.nfy))
    I, J = I.ravel() % n, J.ravel() % n
    ind = m.independent()
    checked = 0
    n_tg3 = 0
    for c in gold:
        alpha = [k for k in range(1, 9) if tuple(d2q9.E[k]) == (c["ex"], c["ey"])][0]
        phi = 2 * np.pi * (c["mx"] * I + c["my"] * J) / n
        u = np.cos(phi)
        f = np.tile(u, (9, 1))
        r = o.advection(f, e, c["C"], 1.0)
        if c["tg3"]:
            x = o.mass_solve(r[alpha - 1], e=(c["ex"], c["ey"]), tg3_coefficient=c["C"] ** 2 / 6)
            n_tg3 += 1
        else:
            x = o.mass_solve(r[alpha - 1])
        up = u + x
        cs, sn = np.cos(phi[ind]), np.sin(phi[ind])
        g_re = np.dot(up[ind], cs) / np.dot(cs, cs)
        g_im = -np.dot(up[ind], sn) / np.dot(sn, sn)
        assert abs(g_re - c["G_re"]) < 1e-12 and abs(g_im - c["G_im"]) < 1e-12, c
        checked += 1
    assert checked >= 120 and n_tg3 >= 60


def test_stencil_bench_check_value(oracle_mod):
    """Q1 lumped streaming increment on a periodic grid reproduces stencil_bench.cc's check value."""
    gold = json.load(open(os.path.join(GOLDEN, "stencil_bench.json")))
    for row in gold["rows"]:
        N = row["N"]
        m = unit_mesh(N, 1, h=1.0 / N)
        o = oracle_mod.Oracle(m, make_params(mass="lumped"))
        I, J = np.meshgrid(np.arange(m.nfx), np.arange(m.nfy))
        idx = (J.ravel() % N) * N + (I.ravel() % N)
        fu = 1.0 + 1e-3 * ((idx * 7919) % 13)
        f = np.tile(fu, (9, 1))
        r = o.advection(f, directions(), 0.25 / N, 1.0, remove_wall_mass_flux=0)
        node = 1 * m.nfx + 1
        chk = sum(o.mass_solve(r[a])[node] for a in range(8))
        assert abs(chk - row["chk"]) <= 5e-6 * abs(row["chk"]), (N, chk, row["chk"])


# ------------------------------------------------------ accuracy tables
def _tgv_error(oracle_mod, N, scheme, mass, p=1):
    tc, m = tgv(N, p=p)
    dt, n = cases.run_length(tc, m, 0.25, 0.25)
    o = setup_case(oracle_mod.Oracle, tc, m, make_params(scheme, mass), dt, tc.relaxation_time())
    o.step(n)
    return cases.diagnostics(tc, m, o.node_weight(), o.get_populations(), n * dt)["rel_l2_u"]


@pytest.mark.parametrize("N,scheme,mass,p,expected", [
    (32, "bardow", "cg", 1, 5.8e-2),
    (32, "leelin", "cg", 1, 6.4e-2),
    (32, "bardow", "lumped", 1, 1.0e-1),
    (64, "bardow", "lumped", 1, 8.8e-3),
    (16, "bardow", "cg", 2, 1.7e-2),
])
def test_tgv_error_table(oracle_mod, N, scheme, mass, p, expected):
    """docs/results.md:54-59 (modes (1,4), Re 100, CFL 0.25, t = t_ref/4, Ma 0.05), to the printed digits."""
    err = _tgv_error(oracle_mod, N, scheme, mass, p)
    assert float(f"{err:.1e}") == expected, err


@pytest.mark.parametrize("N,streaming,cfl,mach,expected,its", [
    (24, "tg3", 0.25, 0.05, 1.49e-1, None),
    (32, "tg3", 0.25, 0.05, 6.16e-2, None),
    (24, "tg3", 1.0, 0.05, 1.04e-1, 5.1),
    (32, "tg3", 1.0, 0.05, 5.00e-2, 4.9),
    (24, "tg3-split", 1.0, 0.05, 3.26e-2, None),
    (32, "tg3-split", 1.0, 0.05, 2.15e-2, None),
    (48, "tg3-split", 1.0, 0.05, 5.75e-3, None),
    (24, "tg3-split", 1.0, 1.6 / 24, 5.38e-2, None),
    (96, "tg2", 0.25, 0.05, 2.89e-3, None),
    (96, "tg3", 1.0, 0.05, 2.84e-3, 2.1),
    (96, "tg3-split", 1.0, 0.05, 2.16e-3, None),
])
def test_tg3_error_table(oracle_mod, N, streaming, cfl, mach, expected, its):
    """docs/results.md:97-107 (TG2 at CFL 0.25, TG3 at CFL 0.25 and 1, with the mean
    CG iterations per solve at CFL 1) and :143-149 (split TG3 at CFL 1, Ma 0.05 and 1.6/N):
    bardow, consistent mass, modes (1,4), Re 100, t = t_ref/4, to the printed digits."""
    tc, m = tgv(N, mach=mach)
    dt, n = cases.run_length(tc, m, cfl, 0.25)
    o = setup_case(oracle_mod.Oracle, tc, m, make_params("bardow", "cg", streaming=streaming), dt,
                   tc.relaxation_time())
    o.step(n)
    err = cases.diagnostics(tc, m, o.node_weight(), o.get_populations(), n * dt)["rel_l2_u"]
    assert float(f"{err:.2e}") == expected, err
    if its is not None:
        solves = n * (12 if streaming == "tg3-split" else 8)
        assert round(o.cg_iterations() / solves, 1) == its


def test_tg3_operator(oracle_mod):
    """A = M + c K_e (mass.h:57-129): symmetric, K_e annihilates functions constant
    along e, and on a uniform periodic Q1 grid at c = h^2/6 along x the x sweep
    operator is I_x (x) M_y (the 1-D matrix (M_x + K_x/6) of a unit CFL is the
    identity times h), so A u = h (I (x) M_y) u."""
    n, h = 8, 1.0 / 8
    m = unit_mesh(n, 1, h=h)
    tc, _ = tgv(n)
    o = setup_case(oracle_mod.Oracle, tc, m, make_params("bardow", "cg", streaming="tg3"), 0.1 * h, 1.0)
    rng = np.random.default_rng(3)
    ind = m.master()
    x, y = m.nodes()
    # symmetry through the solve: r -> x = A^{-1} r with A symmetric => <A^{-1} r1, r2> = <r1, A^{-1} r2>
    e = np.array([1.0, -1.0])
    r1, r2 = rng.standard_normal(m.n_dofs)[ind], rng.standard_normal(m.n_dofs)[ind]
    x1 = o.mass_solve(r1, e=e, tg3_coefficient=0.3 * h * h)
    x2 = o.mass_solve(r2, e=e, tg3_coefficient=0.3 * h * h)
    indep = m.independent()
    assert abs(x1[indep] @ r2[indep] - r1[indep] @ x2[indep]) < 1e-6 * abs(x1[indep] @ r2[indep])  # CG to 1e-8 of |r|
    # unit-CFL x sweep: A u = h (I (x) M_y) u  =>  A^{-1} (h (I (x) M_y) u) = u
    u = np.sin(2 * np.pi * x) * np.cos(4 * np.pi * y) + 0.1 * rng.standard_normal(m.n_dofs)
    u = u[ind]
    nfx = m.nfx
    U = u.reshape(m.nfy, nfx)[:-1, :-1]
    # (I (x) M_y) u on the periodic grid, M_y = h/6 [1 4 1]
    myU = h / 6 * (np.roll(U, 1, 0) + 4 * U + np.roll(U, -1, 0))
    b = np.zeros((m.nfy, nfx))
    b[:-1, :-1] = h * myU
    b[-1, :] = b[0, :]
    b[:, -1] = b[:, 0]
    got = o.mass_solve(b.ravel(), e=np.array([1.0, 0.0]), tg3_coefficient=h * h / 6)
    assert np.max(np.abs(got[indep] - u[indep])) < 1e-6 * np.max(np.abs(u))


def test_tg3_needs_bardow_and_consistent_mass(oracle_mod):
    """streaming.h:51-52 (TG3 needs Mass::cg) and schemes.h:87 (Lee-Lin streams with TG2 only)."""
    tc, m = tgv(8)
    for scheme, mass in (("bardow", "lumped"), ("bardow", "richardson"), ("leelin", "cg")):
        with pytest.raises(LbfemError):
            oracle_mod.Oracle(m, make_params(scheme, mass, streaming="tg3-split"))


def _cavity_golden():
    """data/cavity/cavity_Re1000.dat of the reference (32^2 Q2, stretch 1.2, Ma 0.1):
    its text and its rows x y u/U0 v/U0 psi/(U0 L) rho-rho0."""
    import gzip

    text = gzip.open(os.path.join(GOLDEN, "cavity_Re1000.dat.gz"), "rt").read()
    rows = np.array([ln.split() for ln in text.splitlines() if ln.strip() and not ln.startswith("#")], float)
    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(1000)
    return text, rows, tc, cases.build_mesh(tc, 32, 2)


def test_stream_function_reproduces_the_reference_cavity(oracle_mod):
    """compute_stream_function (io.h:31-95) of the reference's own steady cavity
    velocities gives its printed psi to the print resolution, on the same nodes."""
    text, rows, tc, m = _cavity_golden()
    x, y = m.nodes()
    assert np.max(np.abs(rows[:, 0] - x)) < 1e-6 and np.max(np.abs(rows[:, 1] - y)) < 1e-6
    o = oracle_mod.Oracle(m, make_params("bardow", "lumped"))
    psi = o.stream_function(np.stack([rows[:, 2], rows[:, 3]])) / tc.L
    assert np.max(np.abs(psi - rows[:, 4])) < 1e-6, np.max(np.abs(psi - rows[:, 4]))
    assert np.all(psi[m.constrained() | (x == 0) | (y == 0) | (x == 1) | (y == 1)] == 0)


def test_gnuplot_writer_reproduces_the_reference_cavity_file(oracle_mod):
    """cgdbe.cc:399-472: the same header, row order, blank lines, number format
    and vortex lines as the reference's file, from populations with its moments."""
    from lbfem_gpu import io

    text, rows, tc, m = _cavity_golden()
    o = oracle_mod.Oracle(m, make_params("bardow", "lumped"))
    o.set_time_step(1e-3, 1e-3)
    o.set_populations(d2q9.equilibrium(1 + rows[:, 5], rows[:, 2] * tc.U0, rows[:, 3] * tc.U0))
    out = io.gnuplot_text(o, m, tc, t_over_tref=32.9998, step=391314, reynolds=1000, mach=0.1, n_cells=32)
    a, b = text.splitlines(), out.splitlines()
    assert len(a) == len(b) and a[:2] == b[:2]
    assert [ln == "" for ln in a] == [ln == "" for ln in b]
    same = 0
    for la, lb in zip(a, b):
        if la == lb:
            same += 1
            continue
        va, vb = [float(t) for t in la.split()[-6:] if t[0] in "-.0123456789"], \
                 [float(t) for t in lb.split()[-6:] if t[0] in "-.0123456789"]
        # the last printed digit of psi may differ: the velocities it is solved from are rounded to 6 digits
        assert np.allclose(va, vb, rtol=5e-5, atol=1e-6), (la, lb)
    assert same > 0.8 * len(a)
    assert [ln.split(":")[0] for ln in a[-3:]] == ["# primary vortex", "# lower left vortex", "# lower right vortex"]
    assert a[-3] == b[-3] and a[-1] == b[-1]


def test_cavity_continuation_against_ghia(oracle_mod):
    """The reference's CI check (ci.yml:44-58): cavity, 16^2 Q1, Bardow, lumped mass,
    CFL 0.4, Re 100 to a steady state, then continued to Re 400; psi_max within 10%
    of Ghia, Ghia & Shin (1982): 0.1034 and 0.1139."""
    from lbfem_gpu import driver, io

    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(100)
    m = cases.build_mesh(tc, 16, 1)
    dt = m.time_step(0.4)
    o = setup_case(oracle_mod.Oracle, tc, m, make_params("bardow", "lumped"), dt, tc.relaxation_time())
    for Re, ghia in ((100, 0.1034), (400, 0.1139)):
        if Re != 100:
            tc.set_reynolds(Re)
            o.set_time_step(dt, tc.relaxation_time())
        steps, converged, rate = driver.steady_state(o, m, tc, dt)
        assert converged, (Re, steps, rate)
        text = io.gnuplot_text(o, m, tc, t_over_tref=steps * dt / tc.reference_time(), step=steps, reynolds=Re,
                               mach=0.1, n_cells=16)
        psi_max = float([ln for ln in text.splitlines() if ln.startswith("# primary vortex")][0].split()[5])
        assert abs(psi_max - ghia) <= 0.1 * ghia, (Re, psi_max)


def test_gnuplot_writer_unsteady_rows(oracle_mod):
    """cgdbe.cc:399-446 for an unsteady case: rows x y u/U0 v/U0 |u|/U0 of every
    node (the periodic images with their source's values), grid rows separated by
    blank lines, no vortex lines."""
    from lbfem_gpu import io

    tc, m = tgv(6, p=2)
    o = setup_case(oracle_mod.Oracle, tc, m, make_params("bardow", "cg"), m.time_step(0.25),
                   tc.relaxation_time())
    o.step(3)
    text = io.gnuplot_text(o, m, tc, t_over_tref=0.5, step=3, reynolds=100, mach=0.05, n_cells=6)
    lines = text.splitlines()
    assert lines[0] == "# t/t_ref = 0.5 (step 3), Re = 100, Ma = 0.05, 6^2 Q2 elements"
    assert lines[1] == "# x y u/U0 v/U0 |u|/U0"
    rows = [ln for ln in lines[2:] if ln]
    assert len(rows) == m.n_dofs and lines[2:].count("") == m.nfy - 1
    a = np.array([r.split() for r in rows], float)
    assert a.shape[1] == 5 and np.allclose(a[:, 4], np.hypot(a[:, 2], a[:, 3]), rtol=1e-5, atol=1e-6)
    # the image row y = 1 repeats the row y = 0, the image column x = 1 the column x = 0
    g = a.reshape(m.nfy, m.nfx, 5)
    assert np.array_equal(g[-1, :, 2:], g[0, :, 2:]) and np.array_equal(g[:, -1, 2:], g[:, 0, 2:])


def test_couette_steady_profile(oracle_mod):
    """docs/results.md:253-260: the steady linear profile to solver tolerance (16 elements, Re 10, t = 2 L^2/nu)."""
    tc = cases.CouetteFlow(0.1)
    tc.set_reynolds(10)
    m = cases.build_mesh(tc, 16, 1)
    dt, n = cases.run_length(tc, m, 0.25, 2.0)
    for scheme in ("bardow", "leelin"):
        o = setup_case(oracle_mod.Oracle, tc, m, make_params(scheme, "lumped"), dt, tc.relaxation_time())
        o.step(n)
        d = cases.diagnostics(tc, m, o.node_weight(), o.get_populations(), n * dt)
        assert d["rel_l2_u"] < 1e-9, (scheme, d["rel_l2_u"])
        assert abs(d["mass_drift"]) < 1e-10


def test_cg_no_convergence(oracle_mod):
    """The iteration cap raises NoConvergence (SolverControl, mass.h:38-43)."""
    tc, m = tgv(8)
    o = oracle_mod.Oracle(m, make_params(cg_tolerance=1e-14, cg_max_iterations=1))
    r = np.sin(np.arange(m.n_dofs) * 0.37)
    r[m.constrained()] = 0
    with pytest.raises(_abi.NoConvergence):
        o.mass_solve(r)


def test_cg_zero_rhs_zero_iterations(oracle_mod):
    """A zero right-hand side with a zero start converges at step 0 (tol = 0, |r| = 0)."""
    tc, m = tgv(8)
    o = oracle_mod.Oracle(m, make_params())
    x = o.mass_solve(np.zeros(m.n_dofs))
    assert np.all(x == 0) and o.cg_iterations() == 0


def test_cg_zero_rhs_nonzero_start_gives_zero(oracle_mod):
    """A zero right-hand side with a nonzero start returns the exact solution 0
    with no iterations. deal.II's SolverCG would aim at the tolerance
    cg_tol |b| = 0 from the start and throw NoConvergence at the cap; the
    start-up Couette flow on 32 x 256 Q1 cells meets this case (its x-axis
    populations' right-hand side is round-off, exactly zero in some steps
    after nonzero ones), so the rule is what lets that run finish."""
    tc, m = tgv(8)
    o = oracle_mod.Oracle(m, make_params(cg_max_iterations=5))
    x = o.mass_solve(np.zeros(m.n_dofs), x=1e-20 * np.cos(np.arange(m.n_dofs)))
    assert np.all(x == 0) and o.cg_iterations() == 0


def test_bardow_cavity_conserves_mass(oracle_mod):
    """Bardow with the wall mass flux removed conserves the mean density to round-off with the lumped mass."""
    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(400)
    m = cases.build_mesh(tc, 16, 1)
    o = setup_case(oracle_mod.Oracle, tc, m, make_params("bardow", "lumped"), m.time_step(0.4),
                   tc.relaxation_time())
    c0 = o.conservation()
    o.step(300)
    c1 = o.conservation()
    assert abs(c1[1] / c1[0] - c0[1] / c0[0]) < 1e-13
    assert c1[4] > 0  # the lid has set the fluid in motion


def _checkerboard_amplitude(mesh, f):
    """Amplitude of the (pi, pi) mode of population 1 on the distinct nodes."""
    n = mesh.degree * mesh.n_cells_x
    e = f[1, mesh.independent()].reshape(n, n)
    sign = (-1.0) ** np.add.outer(np.arange(n), np.arange(n))
    return abs(np.mean(e * sign))


@pytest.mark.parametrize("cfl,grows", [(0.5, True), (0.45, False)])
def test_leelin_q1_checkerboard_stability_limit(oracle_mod, cfl, grows):
    """Lee-Lin with the consistent mass on Q1 (TGV 64^2, Re 100) is linearly
    unstable at CFL 0.5 for the checkerboard mode and stable at 0.45. From
    symmetric initial data the mode stays at round-off in FP64, so an unseeded
    run survives; a 1e-7 seed (the size of FP32 rounding) grows by about 1.08
    per step. The reference's own algorithm (CG to 1e-8, schemes.h:92-98) is
    the oracle here."""
    tc = cases.TaylorGreenVortex(0.05 / math.sqrt(d2q9.CS2), 1, 1, shift=(0.25, 0.25), chapman_enskog=False)
    tc.set_reynolds(100)
    m = cases.build_mesh(tc, 64, 1)
    dt, lam = m.time_step(cfl), tc.relaxation_time()
    x, y = m.nodes()
    nfx = m.n_cells_x + 1
    k = np.arange(m.n_dofs)
    f0 = tc.initial_populations(x, y, lam) + 1e-7 * ((-1.0) ** (k % nfx + k // nfx))[None, :]
    o = oracle_mod.Oracle(m, make_params("leelin", "cg", cg_tolerance=1e-8))
    o.set_time_step(dt, lam)
    o.set_initial_populations(f0)
    o.step(100)
    a100 = _checkerboard_amplitude(m, o.get_populations())
    o.step(100)
    a200 = _checkerboard_amplitude(m, o.get_populations())
    if grows:
        assert a200 > 100 * a100 > 0, (a100, a200)
    else:
        assert a200 < a100 < 1e-9, (a100, a200)  # decays from the 1e-7 seed


@pytest.mark.timeout(300)
@pytest.mark.parametrize("cells,grows", [(256, True), (128, False)])
def test_cavity_ladder_first_rung_stability(oracle_mod, cells, grows):
    """The first rung of the continuation ladder (lid-driven cavity, Ma 0.1, Re 100,
    Q2, stretch 1.2, CFL 0.4, Bardow, lumped mass) in the reference's own algorithm:
    on 256^2 cells the peak velocity grows without bound within 100 steps; on
    128^2 it stays at the lid's scale. The ladder runs on 128^2 for this reason."""
    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(100)
    m = cases.build_mesh(tc, cells, 2)
    dt, lam = m.time_step(0.4), tc.relaxation_time()
    x, y = m.nodes()
    o = oracle_mod.Oracle(m, make_params("bardow", "lumped"))
    o.set_time_step(dt, lam)
    o.set_initial_populations(tc.initial_populations(x, y, lam))
    o.step(100)
    _, ux, uy = d2q9.moments(o.get_populations())
    peak = float(np.max(np.hypot(ux, uy)))
    if grows:
        assert peak > 10 * tc.U0, peak
    else:
        assert peak < 2 * tc.U0, peak


def test_checkpoint_format(oracle_mod, tmp_path):
    """write_checkpoint / read_checkpoint (io.h:137-165): name.rank holds the nine
    blocks of Scheme::f one after the other, raw FP64; a torn or foreign file is refused."""
    tc, m = tgv(6, p=2)
    o = setup_case(oracle_mod.Oracle, tc, m, make_params("bardow", "cg"), m.time_step(0.3), tc.relaxation_time())
    o.step(3)
    f = o.get_populations()
    name = str(tmp_path / "state")
    o.write_checkpoint(name, rank=3)
    raw = np.fromfile(name + ".3", dtype=np.float64)
    assert raw.size == 9 * m.n_dofs and np.array_equal(raw.reshape(9, -1), f)
    assert not os.path.exists(name + ".3.tmp")
    (2 * f).tofile(name + ".4")
    o.read_checkpoint(name, rank=4)
    assert np.array_equal(o.get_populations(), 2 * f)
    f[:, :5].tofile(name + ".5")
    with pytest.raises(_abi.LbfemError):
        o.read_checkpoint(name, rank=5)


def test_reynolds_ladder_rungs():
    """The continuation ladder's Reynolds numbers: geometric, ends included."""
    from lbfem_gpu import driver

    re = driver.reynolds_ladder(100.0, 3200.0, 16)
    assert len(re) == 16 and re[0] == 100.0 and abs(re[-1] - 3200.0) < 1e-9
    ratios = np.array(re[1:]) / np.array(re[:-1])
    assert np.allclose(ratios, 32.0 ** (1 / 15), rtol=1e-13)
    assert driver.reynolds_ladder(400.0, 800.0, 1) == [400.0]


def test_ladder_warm_start_on_the_oracle(oracle_mod):
    """batched_ladder's warm start (cgdbe.cc:280-290 keeps Scheme::f from one
    Reynolds number to the next): with every rung at the same Reynolds number and
    the lumped mass (no solver history), rung k, warm-started from rung k - 1 at
    stage k, ends bitwise where rung 0 ends; the steps taken count down by stage."""
    from lbfem_gpu import driver

    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(400)
    m = cases.build_mesh(tc, 8, 1)
    dt, lam = m.time_step(0.4), tc.relaxation_time()
    x, y = m.nodes()
    hs = []
    for k in range(3):
        h = oracle_mod.Oracle(m, make_params("bardow", "lumped"))
        h.set_time_step(dt, lam)
        if k == 0:
            h.set_initial_populations(tc.initial_populations(x, y, lam))
        hs.append(h)
    taken = driver.batched_ladder(hs, 4, batch=False)
    assert taken == [12, 8, 4]
    f0 = hs[0].get_populations()
    for h in hs[1:]:
        assert np.array_equal(h.get_populations(), f0)


@pytest.mark.parametrize("eps,expected", [(0.0, 1.73e-2), (0.02, 1.81e-2), (0.04, 2.07e-2)])
def test_distorted_mesh_error_table(oracle_mod, eps, expected):
    """docs/results.md:222-233, general quadrilaterals (--distort eps, test_cases.h:52-63,
    MappingQ1): 48^2, modes (1,4), Re 100, Ma 0.05, TG2 at nominal CFL 0.25, t = t_ref/4,
    Bardow, consistent mass, Q1, to the printed digits. eps = 0 runs the mapped-vertex
    path on the undistorted vertices."""
    tc, m = tgv(48, distort=eps)
    if eps == 0.0:
        VX, VY = np.meshgrid(m.vertex_x, m.vertex_y)
        m.vertex_xy = np.stack([VX, VY], -1)
    dt, n = cases.run_length(tc, m, 0.25, 0.25)
    o = setup_case(oracle_mod.Oracle, tc, m, make_params("bardow", "cg"), dt, tc.relaxation_time())
    o.step(n)
    err = cases.diagnostics(tc, m, o.node_weight(), o.get_populations(), n * dt)["rel_l2_u"]
    assert float(f"{err:.2e}") == expected, err
    # the mapped cells tile the box: the lumped weights of the distinct nodes add up to its area
    w = o.node_weight()
    assert abs(w[m.independent()].sum() - 1.0) <= 1e-13
