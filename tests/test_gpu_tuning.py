"""The run-time choice of the streaming kernel's tile (lbfem_gpu_tuning): the
three compiled shapes give bitwise the same steps, and a mixed context's first
step times them and keeps the fastest."""
import ctypes as C
import os

import numpy as np
import pytest

from helpers import setup_case
from lbfem_gpu import cases, make_params

pytestmark = pytest.mark.gpu


def _run(tc, m, prm, dt, steps, tune):
    import lbfem_gpu

    old = os.environ.get("LBFEM_TUNE")
    if tune is None:
        os.environ.pop("LBFEM_TUNE", None)
    else:
        os.environ["LBFEM_TUNE"] = tune
    try:
        h = setup_case(lbfem_gpu.Solver, tc, m, prm, dt, tc.relaxation_time())
        h.step(steps)
        shape, ms = C.c_int32(), (C.c_float * 3)()
        h._call("tuning", h.h, C.byref(shape), ms)
        f = h.get_populations()
        h.close()
    finally:
        if old is None:
            os.environ.pop("LBFEM_TUNE", None)
        else:
            os.environ["LBFEM_TUNE"] = old
    return f, shape.value, list(ms)


@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("case,scheme", [("tgv", "leelin"), ("cavity", "bardow")])
def test_tile_shapes_agree_bitwise(gpu_lib, p, case, scheme):
    if case == "tgv":
        tc = cases.TaylorGreenVortex(0.05, 1, 1)
        tc.set_reynolds(100)
        m, cfl = cases.build_mesh(tc, 40, p), 0.5
    else:
        tc = cases.LidDrivenCavity(0.1, 1.2)
        tc.set_reynolds(400)
        m, cfl = cases.build_mesh(tc, 40, p), 0.4
    prm = make_params(scheme, "cg", precision="mixed")
    dt = m.time_step(cfl)
    f0, s0, _ = _run(tc, m, prm, dt, 12, "0")
    f1, s1, _ = _run(tc, m, prm, dt, 12, "alt")
    f2, s2, _ = _run(tc, m, prm, dt, 12, "small")
    assert (s0, s1, s2) == (0, 1, 2)
    assert np.array_equal(f0, f1) and np.array_equal(f0, f2)
    ft, st, ms = _run(tc, m, prm, dt, 12, None)
    assert st in (0, 1, 2) and min(ms) > 0 and ms[st] == min(ms)
    assert np.array_equal(ft, f0)
