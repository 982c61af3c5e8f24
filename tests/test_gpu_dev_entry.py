"""The device-pointer forms of the operators (lbfem_gpu_*_dev) through the C
ABI, on torch device buffers and a torch stream, against the CPU oracle: the
calls a shim makes when it keeps the reference's Scheme::step and its vectors
in device memory (advection.h:49-58, mass.h:185, collision.h:105-168). With
and without a caller DoF numbering. FP64 bar as in the parity tests: relative
L2 <= 1e-12 (operators, solves), <= 1e-14 element-wise (nodal maps)."""
import dataclasses

import numpy as np
import pytest

from helpers import directions, random_populations, rel_l2
from lbfem_gpu import cases, d2q9, make_params

pytestmark = pytest.mark.gpu


def _case(name, p):
    if name == "couette":
        tc = cases.CouetteFlow(0.1)
        tc.set_reynolds(10)
        return cases.build_mesh(tc, 10, p)
    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(400)
    return cases.build_mesh(tc, 9, p)


def _perm(m, permuted):
    """(dof_index, perm, mesh for the context): structured node s is the caller's
    DoF perm[s]; the context's mesh gives its wall nodes by caller DoF."""
    if not permuted:
        return None, np.arange(m.n_dofs), m
    perm = np.random.default_rng(5).permutation(m.n_dofs).astype(np.int64)
    mc = dataclasses.replace(m, wall_dof=perm[m.wall_dof])
    return perm, perm, mc


@pytest.mark.parametrize("permuted", [False, True], ids=["structured", "permuted"])
@pytest.mark.parametrize("name,p", [("couette", 1), ("cavity", 2), ("cavity", 3)])
def test_device_operators_match_the_oracle(gpu_lib, oracle_mod, name, p, permuted):
    import torch

    import lbfem_gpu

    m = _case(name, p)
    dof_index, perm, mc = _perm(m, permuted)
    prm = make_params("leelin", "cg", cg_tolerance=1e-12)
    g = lbfem_gpu.Solver(mc, prm, dof_index=dof_index)
    o = oracle_mod.Oracle(m, prm)
    dev = torch.device("cuda:0")
    s = torch.cuda.Stream(device=dev)
    sp = s.cuda_stream

    def to_dev(a):
        # the caller's numbering: entry perm[k] holds structured node k
        out = np.empty_like(a)
        out[..., perm] = a
        return torch.from_numpy(np.ascontiguousarray(out)).to(dev)

    def from_dev(t):
        return t.cpu().numpy()[..., perm]

    f = random_populations(m, seed=2 * p)
    feq = d2q9.equilibrium(*d2q9.moments(f))
    dt, lam = m.time_step(0.3), 2e-3
    with torch.cuda.stream(s):
        fd, feqd = to_dev(f), to_dev(feq)
        rhs = torch.empty((8, m.n_dofs), dtype=torch.float64, device=dev)
        for kind in ("taylor_galerkin", "leelin"):
            g.advection_dev(fd.data_ptr(), directions(), dt, lam, rhs.data_ptr(), kind=kind,
                            feq=feqd.data_ptr() if kind == "leelin" else 0, stream=sp)
            a = from_dev(rhs)
            b = o.advection(f, directions(), dt, lam, kind=kind, feq=feq if kind == "leelin" else None)
            for al in range(8):
                assert rel_l2(a[al], b[al]) <= 1e-12, (kind, al, rel_l2(a[al], b[al]))
        # the mass solve, from a non-zero start
        r = np.random.default_rng(p).standard_normal(m.n_dofs)
        x0 = 0.1 * np.random.default_rng(p + 1).standard_normal(m.n_dofs)
        xd, rd = to_dev(x0), to_dev(r)
        g.mass_solve_dev(xd.data_ptr(), rd.data_ptr(), stream=sp)
        assert rel_l2(from_dev(xd), o.mass_solve(r, x0)) <= 1e-12
        # nodal maps, in place on the device
        gd = to_dev(f)
        g.collide_bgk_dev(gd.data_ptr(), 1.3, stream=sp)
        b = o.collide_bgk(f, 1.3)
        assert np.max(np.abs(from_dev(gd) - b)) <= 1e-14 * np.max(np.abs(b))
        out = torch.empty_like(fd)
        g.compute_equilibrium_dev(fd.data_ptr(), out.data_ptr(), stream=sp)
        b = o.compute_equilibrium(f)
        assert np.max(np.abs(from_dev(out) - b)) <= 1e-14 * np.max(np.abs(b))
        incr = 1e-3 * np.random.default_rng(p + 2).standard_normal((8, m.n_dofs))
        pd, xi = to_dev(f), to_dev(incr)
        g.predictor_corrector_dev(pd.data_ptr(), feqd.data_ptr(), xi.data_ptr(), 0.7, stream=sp)
        b = o.predictor_corrector(f, feq, incr, 0.7)
        assert np.max(np.abs(from_dev(pd) - b)) <= 1e-14 * np.max(np.abs(b))
    s.synchronize()
    g.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("permuted", [False, True], ids=["structured", "permuted"])
def test_device_populations_and_stream_step(gpu_lib, precision, permuted):
    """set/get_populations_dev and step_stream on a torch stream give what the
    host-buffer calls give (bitwise: the same kernels in the same order)."""
    import torch

    import lbfem_gpu

    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(400)
    m = cases.build_mesh(tc, 12, 2)
    dof_index, perm, mc = _perm(m, permuted)
    prm = make_params("bardow", "cg", precision=precision)
    dt, lam = m.time_step(0.4), tc.relaxation_time()
    x, y = m.nodes()
    f0 = tc.initial_populations(x, y, lam)
    fin = np.empty_like(f0)
    fin[:, perm] = f0
    ref = lbfem_gpu.Solver(mc, prm, dof_index=dof_index)
    ref.set_time_step(dt, lam)
    ref.set_populations(fin)
    ref.step(7)
    expect = ref.get_populations()
    ref.close()
    g = lbfem_gpu.Solver(mc, prm, dof_index=dof_index)
    g.set_time_step(dt, lam)
    dev = torch.device("cuda:0")
    s = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(s):
        fd = torch.from_numpy(fin).to(dev)
        g.set_populations_dev(fd.data_ptr(), stream=s.cuda_stream)
        g.step_stream(7, stream=s.cuda_stream)
        out = torch.full_like(fd, float("nan"))
        g.get_populations_dev(out.data_ptr(), stream=s.cuda_stream)
        got = out.cpu().numpy()  # ordered after the get on the same stream
    s.synchronize()
    assert np.array_equal(got, expect)
    g.close()
