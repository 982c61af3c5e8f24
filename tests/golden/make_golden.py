"""Generates the golden fixtures of tests/golden/ from the reference itself.

Run in a container that has the reference sources, named by $LBFEM_REFERENCE
(required), and the reference program built by `make -C oracle ref`:

    LBFEM_REFERENCE=<lbm-fem tree> python tests/golden/make_golden.py

It writes
  stencils.json       -- assembled stencils of M, C_e, K_e for Q1 and Q2 on a
                         uniform grid, as printed by the reference's
                         analysis/stencils.py (sympy, exact fractions);
  tg_spectral.json    -- amplification factors G_2d of the TG2 / TG3 streaming
                         step from the reference's analysis/tg_spectral.py
                         (imported with a stand-in for matplotlib, which only
                         its plotting code uses);
  stencil_bench.json  -- the check value printed by the reference's
                         benchmarks/stencil_bench.cc (Q1 lumped Lax-Wendroff
                         streaming, periodic N x N grid, dt = h/4) for several N;
  cavity_Re1000.dat.gz -- the reference's own steady cavity result
                         data/cavity/cavity_Re1000.dat (gnuplot rows
                         x y u/U0 v/U0 psi/(U0 L) rho-rho0 of 32^2 Q2 elements,
                         stretch 1.2, and the vortex extrema), gzipped as is.

The fixtures are committed; tests never read the reference at run time.
"""
import importlib.util
import json
import os
import re
import subprocess
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("LBFEM_REFERENCE")
if not REF:
    sys.exit("make_golden.py: set LBFEM_REFERENCE to the lbm-fem source tree")


def load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_stencils():
    import sympy as sp

    st = load("ref_stencils", os.path.join(REF, "analysis", "stencils.py"))
    out = {}
    for p in (1, 2):
        for name, e in (("(1,0)", (1, 0)), ("(1,1)", (1, 1)), ("(0,1)", (0, 1)), ("(-1,1)", (-1, 1))):
            M, Cm, K, X = st.element_matrices(p, e)
            for label, A in (("M", M), ("C", Cm), ("K", K)):
                key = f"Q{p} {label}" + ("" if label == "M" else f" e={name}")
                if key in out:
                    continue
                table = {}
                for node, s in st.stencils(p, A, X).items():
                    # values at h = 1 (M scales h^2, C h, K h^0 on a square h x h element)
                    table[f"{int(node[0])},{int(node[1])}"] = {
                        f"{int(k[0])},{int(k[1])}": float(sp.nsimplify(v).subs(st.h, 1)) for k, v in s.items()
                    }
                out[key] = table
    return out


def make_tg_spectral():
    import numpy as np

    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    pyplot = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = pyplot
    saved = {k: sys.modules.get(k) for k in ("matplotlib", "matplotlib.pyplot")}
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = pyplot
    try:
        tg = load("ref_tg_spectral", os.path.join(REF, "analysis", "tg_spectral.py"))
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    cases = []
    n = 16
    for mx, my in ((1, 0), (0, 2), (1, 1), (3, 1), (2, 5), (5, 3)):
        tx, ty = 2 * np.pi * mx / n, 2 * np.pi * my / n
        for e in ((1, 0), (0, 1), (1, 1), (-1, 1), (-1, -1), (1, -1)):
            for C in (0.1, 0.25):
                for tg3 in (False, True):
                    G = complex(tg.G_2d(tx, ty, e[0], e[1], C, tg3))
                    cases.append({"n": n, "mx": mx, "my": my, "ex": e[0], "ey": e[1], "C": C, "tg3": tg3,
                                  "G_re": G.real, "G_im": G.imag})
    return {"source": "analysis/tg_spectral.py G_2d", "cases": cases}


def make_stencil_bench():
    exe = os.path.join(REPO, "oracle", "_ref", "stencil_bench")
    if not os.path.exists(exe):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "ref", f"REFERENCE={REF}"], check=True)
    rows = []
    for N in (16, 24, 32, 48, 64):
        txt = subprocess.run([exe, str(N)], check=True, capture_output=True, text=True).stdout
        chk = float(re.search(r"chk ([-+0-9.eE]+)\)", txt).group(1))
        rows.append({"N": N, "chk": chk})
    return {"source": "benchmarks/stencil_bench.cc: chk = sum_{a=1..8} r_a at node (1,1); printed %g",
            "dt_over_h": 0.25, "rows": rows}


def copy_cavity(name="cavity_Re1000.dat"):
    import gzip

    with open(os.path.join(REF, "data", "cavity", name), "rb") as src:
        data = src.read()
    with gzip.GzipFile(os.path.join(HERE, name + ".gz"), "wb", mtime=0) as dst:
        dst.write(data)
    print("wrote", name + ".gz")


if __name__ == "__main__":
    copy_cavity()
    for name, fn in (("stencils.json", make_stencils), ("tg_spectral.json", make_tg_spectral),
                     ("stencil_bench.json", make_stencil_bench)):
        with open(os.path.join(HERE, name), "w") as fh:
            json.dump(fn(), fh, indent=1, sort_keys=True)
        print("wrote", name)
