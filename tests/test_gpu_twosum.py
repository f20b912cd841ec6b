"""The TwoSum-compensated FP32 row accumulator (AED_FP32_ACCUM=twosum; needs a B200).

The accumulator is chosen once per process from the environment, so the
checks run in a child process: FP32 rows of every apply variant within
2 eps32 * sum_j |M_ij x_j| of the explicit matrix's exact rows (the same bound
as the default FP64-accumulator rows), and a mixed-precision solve within
1e-9 of the FP64 solve.
"""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import alps_b200 as ed
import oracle
from oracle import lattice

out = {}
eps = float(np.finfo(np.float32).eps)
for name, lat, prm, seed in [("square4x5", "square lattice", {"L": 4, "W": 5}, 3),
                             ("nnn18", "nnn chain lattice", {"L": 18}, 4)]:
    n, _, raw = lattice.lattice_graph(lat, prm)
    js = np.random.default_rng(seed).uniform(0.5, 1.5, len(raw))
    bonds = [(s, t, float(j), float(j), 0.0) for (s, t, _), j in zip(raw, js)]
    ham = ed.Hamiltonian(n, n // 2, bonds, precision=ed.FP32)
    M = oracle.Matrix(n, n // 2, bonds)
    rp, col, val = M.csr()
    x = np.random.default_rng(seed).normal(size=ham.dim).astype(np.float32).astype(np.float64)
    ref = M.mult(x)
    absrow = np.add.reduceat(np.abs(val) * np.abs(x[col]), rp[:-1])
    xd, yd = ham.new_vector().upload(x), ham.new_vector()
    worst = 0.0
    nvar = 0
    for v in range(len(ed.apply_variants())):
        try:
            ham.time_apply(xd, yd, 1, v)
        except ed.AEDError:
            continue
        nvar += 1
        y = yd.download()
        worst = max(worst, float(np.max(np.abs(y - ref) / (2 * eps * absrow + 1e-300))))
    r64 = ed.Hamiltonian(n, n // 2, bonds).solve(nev=2, seed=7)
    r32 = ham.solve(nev=2, seed=7)
    rel = float(np.max(np.abs(r32["evals"] - r64["evals"]) / np.abs(r64["evals"])))
    out[name] = {"worst_over_bound": worst, "variants": nvar, "rel": rel,
                 "n64": len(r64["evals"]), "n32": len(r32["evals"])}
print(json.dumps(out))
"""


def test_twosum_accumulator_rows_and_mixed_solve():
    env = dict(os.environ, AED_FP32_ACCUM="twosum")
    p = subprocess.run([sys.executable, "-c", CHILD, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    res = json.loads(p.stdout.strip().splitlines()[-1])
    for name, r in res.items():
        assert r["variants"] >= 1, name
        assert r["worst_over_bound"] <= 1.0, (name, r)
        assert r["n32"] == r["n64"] and r["rel"] <= 1e-9, (name, r)
