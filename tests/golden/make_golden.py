"""Generate the golden fixtures in this folder from the reference project's own code.

Run in a container where the reference source tree is mounted (default
``/root/reference``; override with ``HASTY_REFERENCE``):

    python tests/golden/make_golden.py

What it produces (``golden_ahwa.npz``):

* ``coords``: the fixed sample table of ``lib/tests/tests1.cpp:73-174`` (used by
  ``test_deterministic_3d`` and ``compare_normal_methods``), mapped exactly as the
  reference maps it (``tests1.cpp:176-180``): ``-pi + 2*pi*u`` rounded to float32.
* For each case: an input image ``x_<case>`` and ``y_<case> = (A^H W A) x`` computed by
  the reference's own dense builder ``compute_AHWA`` /
  ``compute_AHWA_element`` / ``expi``
  (``python/python/hastypy/tests/toepbuilder/toep_builder.py:24-82``), executed from
  the reference source.  That module runs plotting/torchkbnufft code at import, so
  only those three function definitions are extracted with ``ast`` and executed with
  ``numba.njit`` replaced by the identity (numba is not installed here).

Cases:
* ``cnm``: the ``compare_normal_methods`` case (``tests1.cpp:351-549``): a ones image of
  shape (nz, ny, nx) = (3, 2, 5) and the first 30 fixed samples.
* ``rnd``: a seeded complex image of shape (4, 3, 5) and all 100 fixed samples.

The oracle's Toeplitz normal operator times prod(2N) and its explicit normal operator
times prod(N) must both equal ``y`` (see ``tests/test_oracle.py``).
"""
from __future__ import annotations

import ast
import os
import re
import sys

import numpy as np

REF = os.environ.get("HASTY_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))


def read_fixed_coords():
    path = os.path.join(REF, "lib", "tests", "tests1.cpp")
    with open(path) as f:
        lines = f.readlines()
    # first table: lines 73-174 (1-based) of tests1.cpp
    body = "".join(lines[72:174])
    rows = re.findall(r"\{\s*([-0-9.eE]+)\s*,\s*([-0-9.eE]+)\s*,\s*([-0-9.eE]+)\s*\}", body)
    u = np.array([[float(a) for a in r] for r in rows], dtype=np.float64)
    assert u.shape == (100, 3), u.shape
    u32 = u.astype(np.float32)  # std::array<float,3> literals
    # coords.index_put_({a,l}, -M_PI + 2*M_PI*fixed[l][a]) : double math, stored as float32
    coords = (-np.pi + 2 * np.pi * u32.astype(np.float64)).astype(np.float32)
    return coords.T.copy()  # [3, 100]


def load_ahwa_functions(nf):
    path = os.path.join(REF, "python", "python", "hastypy", "tests", "toepbuilder", "toep_builder.py")
    with open(path) as f:
        src = f.read()
    tree = ast.parse(src)
    wanted = {"expi", "compute_AHWA_element", "compute_AHWA"}
    defs = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in wanted]
    assert {d.name for d in defs} == wanted
    mod = ast.Module(body=defs, type_ignores=[])
    ns = {"np": np, "njit": (lambda f: f), "nf": nf}
    exec(compile(mod, path, "exec"), ns)
    return ns


def main():
    coords_all = read_fixed_coords()
    out = {"coords": coords_all}
    rng = np.random.default_rng(20261203)
    cases = {
        "cnm": (np.ones((3, 2, 5), np.complex128), 30),
        "rnd": (rng.standard_normal((4, 3, 5)) + 1j * rng.standard_normal((4, 3, 5)), 100),
    }
    for name, (x, nf) in cases.items():
        ns = load_ahwa_functions(nf)
        c = coords_all[:, :nf].astype(np.float64)
        w = np.ones(nf, np.float64)
        y = ns["compute_AHWA"](c, w, x)
        out[f"x_{name}"] = x
        out[f"y_{name}"] = np.asarray(y, np.complex128)
        out[f"nf_{name}"] = np.int64(nf)
        print(name, x.shape, nf, np.abs(y).max(), file=sys.stderr)
    np.savez_compressed(os.path.join(HERE, "golden_ahwa.npz"), **out)


if __name__ == "__main__":
    main()
