"""include/aed_ietl.hpp driven as ietl::lanczos drives its MATRIX / VS (C++, through the C ABI)."""

import os
import subprocess

import numpy as np
import pytest

import oracle
from oracle import lattice

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def adaptor_binary(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "ietl_adaptor_check")
    lib = os.path.join(ROOT, "alps_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "ietl_adaptor_check.cpp"), "-L" + lib, "-laed",
                    "-Wl,-rpath," + lib, "-o", out], check=True)
    return out


def test_ietl_recurrence_through_adaptor_matches_oracle(adaptor_binary):
    steps = 25
    res = subprocess.run([adaptor_binary, "16", str(steps), "1"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stderr
    ab = np.array([[float(v) for v in line.split()] for line in res.stdout.strip().splitlines()])
    assert ab.shape == (steps, 2)
    N, nu, bonds = lattice.spin_model({"LATTICE": "chain lattice", "L": 16, "J": 1, "Sz_total": 0})
    o = oracle.Matrix(N, nu, bonds).lanczos(nev=4, seed=1)
    np.testing.assert_allclose(ab[:, 0], o["alpha"][:steps], rtol=1e-9)
    np.testing.assert_allclose(ab[:, 1], o["beta"][:steps], rtol=1e-8)
