"""Ritz vectors (aed_eigenvectors) and checkpoint / resume of the Lanczos recurrence
(aed_lanczos_save / aed_lanczos_load / aed_solve with resume), through the C ABI (needs a B200)."""

import numpy as np
import pytest

import alps_b200 as ed
import oracle

pytestmark = pytest.mark.gpu


def random_chain(L, seed, j2=0.3):
    """J1-J2 chain with per-bond couplings and a small field: no degenerate levels."""
    rng = np.random.default_rng(seed)
    bonds = []
    for i in range(L):
        j1 = rng.uniform(0.8, 1.2)
        bonds.append((i, (i + 1) % L, j1, j1))
        jj = j2 * rng.uniform(0.8, 1.2)
        bonds.append((i, (i + 2) % L, jj, jj))
    h = rng.uniform(-0.1, 0.1, L).tolist()
    return bonds, h


def dense_spectrum(L, bonds, h):
    M = oracle.Matrix(L, L // 2, bonds, site_h=h)
    w, V = np.linalg.eigh(M.dense())
    return M, w, V


@pytest.mark.parametrize("prec", [ed.FP64, ed.FP32])
def test_eigenvectors_match_dense(prec):
    L = 14
    bonds, h = random_chain(L, 11)
    M, w, V = dense_spectrum(L, bonds, h)
    ham = ed.Hamiltonian(L, L // 2, bonds, precision=prec, site_h=h)
    r = ham.solve(nev=3, seed=4)
    vecs, ev, res = ham.eigenvectors(3, seed=4)
    np.testing.assert_allclose(ev, r["evals"], rtol=0, atol=0)
    # FP64: the ietl rule leaves residuals near 100 eps |lambda|; mixed: the refinement stops at
    # r^2 / gap <= 1e-11 |lambda| (r ~ 1e-6 here) and the vectors come back rounded to FP32
    fp64 = prec == ed.FP64
    for i in range(3):
        psi = vecs[i].download()
        assert abs(np.linalg.norm(psi) - 1.0) < (1e-12 if fp64 else 1e-6)
        assert abs(abs(psi @ V[:, i]) - 1.0) < (1e-10 if fp64 else 1e-6)
        assert res[i] < (1e-9 if fp64 else 1e-4)
        if fp64:  # the residual reported is |H psi - lambda psi|
            assert abs(np.linalg.norm(M.mult(psi) - ev[i] * psi) - res[i]) < 1e-12
        np.testing.assert_allclose(ev[i], w[i], rtol=1e-11 if fp64 else 1e-9)


def test_eigenvectors_need_the_solves_start():
    L = 12
    bonds, h = random_chain(L, 3)
    ham = ed.Hamiltonian(L, L // 2, bonds, site_h=h)
    ham.solve(nev=2, seed=4)
    with pytest.raises(ed.AEDError) as e:
        ham.eigenvectors(2, seed=5)
    assert e.value.code == ed.ERR_MISMATCH
    with pytest.raises(ed.AEDError):
        ham.eigenvectors(2000, seed=4)  # more than the distinct values found (T is at most D = 924)


def test_checkpoint_resume_continues_the_same_recurrence():
    """Solve for 1 value, save; a fresh handle loads it and resumes for 3: the same T, the same
    eigenvalues, bit for bit, as a direct 3-value solve from the same start."""
    L = 16
    bonds, h = random_chain(L, 7)
    h1 = ed.Hamiltonian(L, L // 2, bonds, site_h=h)
    r1 = h1.solve(nev=1, seed=3)
    state = h1.lanczos_save()
    h2 = ed.Hamiltonian(L, L // 2, bonds, site_h=h)
    h2.lanczos_load(state)
    r2 = h2.solve(nev=3, resume=True)
    h3 = ed.Hamiltonian(L, L // 2, bonds, site_h=h)
    r3 = h3.solve(nev=3, seed=3)
    assert r2["iterations"] > r1["iterations"]
    assert r2["iterations"] == r3["iterations"]
    assert np.array_equal(r2["evals"], r3["evals"])
    a2, b2 = h2.last_tmatrix()
    a3, b3 = h3.last_tmatrix()
    assert np.array_equal(a2, a3) and np.array_equal(b2, b3)
    # the resumed recurrence replays from the original start for its Ritz vectors
    vecs, ev, res = h2.eigenvectors(3, seed=3)
    assert np.array_equal(ev, r3["evals"]) and np.all(res < 1e-9)
    # resuming the handle's own live recurrence works as well
    r4 = h1.solve(nev=3, resume=True)
    assert np.array_equal(r4["evals"], r3["evals"])


def test_checkpoint_rejects_other_models_and_truncation():
    L = 12
    bonds, h = random_chain(L, 5)
    h1 = ed.Hamiltonian(L, L // 2, bonds, site_h=h)
    with pytest.raises(ed.AEDError):  # nothing to save before a solve
        h1.lanczos_save()
    with pytest.raises(ed.AEDError):  # nothing to resume
        h1.solve(nev=1, resume=True)
    h1.solve(nev=1, seed=2)
    state = h1.lanczos_save()
    other, _ = random_chain(L, 6)
    h2 = ed.Hamiltonian(L, L // 2, other, site_h=h)
    with pytest.raises(ed.AEDError):
        h2.lanczos_load(state)
    h3 = ed.Hamiltonian(L, L // 2, bonds, site_h=h)
    with pytest.raises(ed.AEDError):
        h3.lanczos_load(state[: len(state) // 2])
    with pytest.raises(ed.AEDError):
        h3.lanczos_load(b"x" * len(state))
    h3.lanczos_load(state)
    assert h3.solve(nev=1, resume=True)["converged"]
    # new couplings on a handle drop its recurrence
    h1.set_couplings(other)
    with pytest.raises(ed.AEDError):
        h1.solve(nev=1, resume=True)
