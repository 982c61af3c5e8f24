"""The mass solve for callers that cannot allocate device memory when they call
in (lbfem_gpu_mass_solve_noalloc): it must give what the ordinary
lbfem_gpu_mass_solve gives on the same inputs, call after call, although its
CG work buffers live in one fixed device array of the library and the caller
hands in device buffers. The test allocates those device buffers itself (with
torch); the entry point allocates nothing.

Kept in a file of its own that pytest collects last."""
import ctypes as C

import numpy as np
import pytest

from helpers import rel_l2
from lbfem_gpu import _abi, cases, make_params

pytestmark = pytest.mark.gpu


def _solve_noalloc(lib, handle, x_dev, r_dev):
    fn = lib.lbfem_gpu_mass_solve_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    return fn(handle.h, C.c_void_p(x_dev.data_ptr()), C.c_void_p(r_dev.data_ptr()))


def _case(name):
    if name == "cavity":
        tc = cases.LidDrivenCavity(0.1, 1.2)
        tc.set_reynolds(400)
        return cases.build_mesh(tc, 12, 2)
    tc = cases.TaylorGreenVortex(0.05, 1, 4)
    tc.set_reynolds(100)
    return cases.build_mesh(tc, 20, 1)


@pytest.mark.parametrize("name", ["cavity", "tgv"])
def test_noalloc_mass_solve_matches_the_allocating_one(gpu_lib, name):
    import torch

    import lbfem_gpu

    mesh = _case(name)
    h = lbfem_gpu.Solver(mesh, make_params(mass="cg", cg_tolerance=1e-13))
    rng = np.random.default_rng(42)
    for call in range(2):  # two calls in a row: the shared work array is reused
        r = rng.standard_normal(mesh.n_dofs)
        r[mesh.constrained()] = 0
        x0 = 0.05 * rng.standard_normal(mesh.n_dofs)
        x0[mesh.constrained()] = 0
        expected = h.mass_solve(r, x=x0)
        x_dev = torch.tensor(x0, dtype=torch.float64, device="cuda:0")
        r_dev = torch.tensor(r, dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        st = _solve_noalloc(gpu_lib, h, x_dev, r_dev)
        assert st == _abi.LBFEM_OK, gpu_lib.lbfem_gpu_last_error(h.h)
        got = x_dev.cpu().numpy()
        assert rel_l2(got, expected) <= 1e-12, (call, rel_l2(got, expected))
    h.close()


def test_noalloc_rejects_meshes_beyond_its_fixed_size(gpu_lib):
    import torch

    import lbfem_gpu

    tc = cases.TaylorGreenVortex(0.05, 1, 1)
    tc.set_reynolds(100)
    mesh = cases.build_mesh(tc, 400, 1)  # 401^2 = 160801 nodes > 131072
    h = lbfem_gpu.Solver(mesh, make_params(mass="cg"))
    x_dev = torch.zeros(4, dtype=torch.float64, device="cuda:0")
    st = _solve_noalloc(gpu_lib, h, x_dev, x_dev)
    assert st == _abi.LBFEM_ERR_ARG
    assert b"exceed" in gpu_lib.lbfem_gpu_last_error(h.h)
    h.close()
