"""Finishing sums folded into the update and normalisation kernels (needs a B200).

For sectors with short partial lists every CTA of the update sums the
apply's alpha partials itself, and every CTA of the normalisation the beta
partials, in the one-CTA finishing kernel's order.  The choice is made once
per process (AED_FOLD_FINISH=0 keeps the separate kernels), so two child
processes solve the same requests, and alpha, beta, the eigenvalues and the
iteration counts must agree bit for bit.
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
sys.path.insert(0, sys.argv[1])
import alps_b200 as ed

out = {}
for name, n, bonds, prec in [
        ("chain18_fp64", 18, [(i, (i + 1) % 18, 1.0, 1.0, 0.0) for i in range(18)], ed.FP64),
        ("nnn20_mixed", 20, [(i, (i + 1) % 20, 1.0, 1.0, 0.0) for i in range(20)]
                            + [(i, (i + 2) % 20, 0.3, 0.3, 0.0) for i in range(20)], ed.FP32)]:
    ham = ed.Hamiltonian(n, n // 2, bonds, precision=prec)
    r = ham.solve(nev=2, seed=5)
    a, b = ham.last_tmatrix()
    out[name] = {"evals": [float(v).hex() for v in r["evals"]], "iterations": r["iterations"],
                 "iterations_low": r["iterations_low"], "alpha": [float(v).hex() for v in a],
                 "beta": [float(v).hex() for v in b]}
    if prec == ed.FP32:
        a32, b32 = ham.last_tmatrix(fp32_phase=True)
        out[name]["alpha32"] = [float(v).hex() for v in a32]
        out[name]["beta32"] = [float(v).hex() for v in b32]
print(json.dumps(out))
"""


def _run(fold):
    env = dict(os.environ)
    env.pop("AED_FOLD_FINISH", None)
    if not fold:
        env["AED_FOLD_FINISH"] = "0"
    p = subprocess.run([sys.executable, "-c", CHILD, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_folded_finishing_sums_are_bit_identical():
    folded, separate = _run(True), _run(False)
    assert folded.keys() == separate.keys()
    for name in folded:
        assert folded[name] == separate[name], name
        assert len(folded[name]["alpha"]) > 10
