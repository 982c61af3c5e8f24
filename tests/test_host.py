"""CPU checks of the boundary and the host-side set-up: the C-ABI library loads
and exports every symbol include/lbfem_gpu.h declares (no compute call needs
a GPU here), its defaults are the reference's, and the test-case set-up
(mesh, walls, time step) follows test_cases.h / discretization.h."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from lbfem_gpu import _abi, cases


def header_functions():
    text = open(os.path.join(ROOT, "include", "lbfem_gpu.h")).read()
    return sorted(set(re.findall(r"\b(lbfem_gpu_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import lbfem_gpu

    lib = lbfem_gpu.library()
    names = header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_defaults():
    import lbfem_gpu

    lib = lbfem_gpu.library()
    for s in range(8):
        assert lib.lbfem_gpu_status_string(s)
    p = _abi.Params()
    lib.lbfem_gpu_default_params.restype = None
    lib.lbfem_gpu_default_params(C.byref(p))
    # MassSettings / StreamingSettings defaults (mass.h:33-48, streaming.h:32-36), Bardow (cgdbe.cc:65)
    assert (p.scheme, p.mass, p.richardson, p.streaming, p.cg_max_iterations) == (1, 0, 2, 0, 200)
    assert p.cg_tolerance == 1e-8 and p.remove_wall_mass_flux == -1


def test_no_gpu_fails_loudly():
    import lbfem_gpu

    if lbfem_gpu.device_count() > 0:
        pytest.skip("a GPU is present")
    tc = cases.TaylorGreenVortex(0.1, 1, 1)
    tc.set_reynolds(100)
    with pytest.raises(_abi.LbfemError) as ei:
        lbfem_gpu.Solver(cases.build_mesh(tc, 4, 1), lbfem_gpu.make_params())
    assert ei.value.status == _abi.LBFEM_ERR_CUDA


def test_meshes_of_2_31_nodes_are_refused():
    """The kernels index a population array with 32-bit storage indices: create
    refuses a mesh of 2^31 or more nodes before it touches the device."""
    import lbfem_gpu

    lib = lbfem_gpu.library()
    for p, n in ((4, 11586), (1, 46341)):
        vx = np.arange(n + 1, dtype=np.float64)
        nd = (p * n + 1) ** 2
        assert nd >= 2 ** 31
        desc = _abi.MeshDesc(p, n, n, 1, 1, vx.ctypes.data_as(C.POINTER(C.c_double)),
                             vx.ctypes.data_as(C.POINTER(C.c_double)), nd, None, 0, None, None)
        prm = lbfem_gpu.make_params()
        h = C.c_void_p()
        assert lib.lbfem_gpu_create(C.byref(desc), C.byref(prm), C.byref(h)) == _abi.LBFEM_ERR_UNSUPPORTED
        assert not h.value


def test_gauss_lobatto_points_match_oracle(oracle_mod):
    for p in (1, 2, 3, 4):
        s, _, _ = oracle_mod.basis_1d(p)
        assert np.allclose(cases.gauss_lobatto(p), s, atol=1e-15)


def test_cavity_walls_and_time_step():
    tc = cases.LidDrivenCavity(0.1, 1.2)
    tc.set_reynolds(400)
    m = cases.build_mesh(tc, 8, 2)
    x, y = m.nodes()
    # every boundary node is a wall; the lid moves except at its corners (test_cases.h:310-323)
    on = (x < 1e-12) | (x > 1 - 1e-12) | (y < 1e-12) | (y > 1 - 1e-12)
    assert set(m.wall_dof) == set(np.nonzero(on)[0])
    moving = m.wall_dof[m.wall_velocity[:, 0] > 0]
    assert np.all(y[moving] > 1 - 1e-12) and np.all((x[moving] > 1e-12) & (x[moving] < 1 - 1e-12))
    # h_min is the clustered first cell; dt = cfl h_min / p^2 (discretization.h:158-162)
    assert abs(m.h_min - (m.vertex_x[1] - m.vertex_x[0])) < 1e-15
    assert abs(m.time_step(0.4) - 0.4 * m.h_min / 4) < 1e-18


def test_couette_walls_include_periodic_images():
    tc = cases.CouetteFlow(0.1)
    tc.set_reynolds(10)
    m = cases.build_mesh(tc, 4, 1)
    assert len(m.wall_dof) == 2 * m.nfx  # both rows, images included (the reference tags by coordinate)
    assert m.constrained().sum() == m.nfy


def test_run_length_hits_t_end():
    tc = cases.TaylorGreenVortex(0.05, 1, 4)
    tc.set_reynolds(100)
    m = cases.build_mesh(tc, 32, 1)
    dt, n = cases.run_length(tc, m, 0.25, 0.25)
    assert n == 166 and abs(n * dt - 0.25 * tc.reference_time()) < 1e-12


def test_noalloc_tile_bound_is_implied_by_the_node_bound():
    """lbfem_gpu_mass_solve_noalloc's fixed array holds the vectors of at most
    NOALLOC_MAX_NODES nodes and the partial sums of NOALLOC_MAX_TILES tiles. No
    mesh under the node limit has more tiles than the array holds, for every
    degree's tile shape (kernels.cuh TileShape<P>), so the node limit is the
    only one a caller meets."""
    csrc = os.path.join(ROOT, "lbm-fem_b200", "csrc")
    kern = open(os.path.join(csrc, "kernels.cuh")).read()
    src = open(os.path.join(csrc, "lbfem_gpu.cu")).read()
    max_nodes = 1 << int(re.search(r"NOALLOC_MAX_NODES = 1LL << (\d+)", src).group(1))
    max_tiles = int(re.search(r"NOALLOC_MAX_TILES = (\d+)", src).group(1))
    assert (max_nodes, max_tiles) == (131072, 4096)
    shapes = {int(p): (int(cx), int(cy)) for p, cx, cy in re.findall(
        r"struct TileShape<(\d)>\s*\{\s*static constexpr int CX = (\d+), CY = (\d+)", kern)}
    assert sorted(shapes) == [1, 2, 3, 4]
    worst = {}
    for p, (cx, cy) in shapes.items():
        tx, ty = p * cx, p * cy
        most = 0
        for ncx in range(1, max_nodes):
            nfx = p * ncx + 1
            if nfx * (p + 1) > max_nodes:
                break
            # the most cells along y that keep the mesh within the node limit
            nfy = p * ((max_nodes // nfx - 1) // p) + 1
            # both orientations of the box
            most = max(most, -(-nfx // tx) * -(-nfy // ty), -(-nfy // tx) * -(-nfx // ty))
        worst[p] = most
    assert worst[1] == 2731 and max(worst.values()) < max_tiles, worst


def test_mt19937_64_matches_the_cpp_engine(tmp_path):
    """The batched workload's generator reproduces std::mt19937_64(20261203)
    (compiled here with the system C++ compiler): the first 1000 outputs."""
    import shutil
    import subprocess

    import bench

    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "mt.cc"
    src.write_text("#include <cstdio>\n#include <random>\nint main(){std::mt19937_64 g(20261203ULL);"
                   "for(int i=0;i<1000;++i)std::printf(\"%llu\\n\",(unsigned long long)g());}\n")
    exe = tmp_path / "mt"
    subprocess.run([cxx, "-O1", "-o", str(exe), str(src)], check=True)
    want = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    rng = bench.MT19937_64(20261203)
    assert [rng() for _ in range(1000)] == want
    inst = bench.batch_instances(64)
    assert sum(i["case"] == "cavity" for i in inst) == 32
    assert all(100 <= i["Re"] <= 1000 and 0.05 <= i["U0"] <= 0.1 for i in inst)


def _element_matrices(p):
    """FE_Q(p) on [0, 1] at the Gauss-Lobatto points: mass, derivative and
    stiffness matrices by exact Gauss quadrature (numpy, independent of the
    library's geometry code)."""
    x = cases.gauss_lobatto(p)
    n = p + 1
    coef = np.linalg.inv(np.vander(x, n, increasing=True))  # l_a(t) = sum_k coef[k, a] t^k
    g, w = np.polynomial.legendre.leggauss(n + 1)
    t, w = (g + 1) / 2, w / 2
    l = np.vander(t, n, increasing=True) @ coef
    dv = np.zeros((len(t), n))
    for k in range(1, n):
        dv[:, k] = k * t ** (k - 1)
    dl = dv @ coef
    return [(l * w[:, None]).T @ l, (l * w[:, None]).T @ dl, (dl * w[:, None]).T @ dl]


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_fp32_element_matrices_annihilate_constants(p):
    """The FP32 element matrices of the FP32 kernels: the mass matrix is the
    FP64 one rounded; the derivative and stiffness rows sum exactly to zero (their
    plain FP32 roundings do not from p = 2 on), each entry within 1.2e-7 of its
    row's largest."""
    import lbfem_gpu

    lib = lbfem_gpu.library()
    fn = lib.lbfem_gpu_reference_matrix
    fn.restype, fn.argtypes = C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_float)]
    exact = _element_matrices(p)
    n = p + 1
    for op in range(3):
        r64 = np.zeros(n * n)
        r32 = np.zeros(n * n, dtype=np.float32)
        assert fn(p, op, r64.ctypes.data_as(C.POINTER(C.c_double)), r32.ctypes.data_as(C.POINTER(C.c_float))) == 0
        r64, r32 = r64.reshape(n, n), r32.reshape(n, n)
        assert np.allclose(r64, exact[op], rtol=0, atol=1e-13 * np.abs(exact[op]).max())
        tiny = np.abs(r64) <= 1e-14 * np.abs(r64).max(axis=1, keepdims=True)  # exact zeros but for rounding
        if op == 0:
            assert np.array_equal(r32, np.where(tiny, 0.0, r64).astype(np.float32))
            continue
        assert np.all(r32[tiny] == 0)
        for a in range(n):
            row = [float(v) for v in r32[a]]
            assert sum(row) == 0.0  # exact in FP64: a few FP32 values
            assert np.abs(r32[a].astype(np.float64) - r64[a]).max() <= 1.2e-7 * np.abs(r64[a]).max()
    assert fn(0, 0, None, None) != 0 and fn(p, 3, None, None) != 0
