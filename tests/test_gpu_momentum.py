"""Momentum (Bloch) sectors of the CUDA engine against the oracle's restatement (needs a B200)."""

import numpy as np
import pytest

import alps_b200 as ed
from alps_b200 import sparsediag
from oracle import bloch, lattice

pytestmark = pytest.mark.gpu

CASES = [
    ("chain lattice", {"L": 10}, {0: (1.0, 1.0)}),
    ("nnn chain lattice", {"L": 10}, {0: (1.0, 1.0), 1: (0.45, 0.45)}),
    ("square lattice", {"L": 4, "W": 3}, {0: (1.0, 0.8)}),
    ("ladder", {"L": 6}, {0: (1.0, 1.0), 1: (0.6, 0.7)}),
    ("anisotropic square lattice", {"L": 4, "W": 2}, {0: (1.0, 1.2), 1: (0.5, 0.3)}),
]


def _params(lat, geo):
    return dict(geo, MODEL="spin", LATTICE=lat, CONSERVED_QUANTUMNUMBERS="Sz")


def _bonds(lat, geo, coup):
    n, _, graph = lattice.lattice_graph(lat, geo)
    return n, [(s, t, coup[ty][0], coup[ty][1], 0.0) for s, t, ty in graph]


def _sectors(lat, geo, coup, n_ups=None):
    n, bonds = _bonds(lat, geo, coup)
    p = _params(lat, geo)
    for n_up in (n_ups if n_ups is not None else (n // 2, n // 2 - 1)):
        for k in ed.lattice_momenta(p):
            tr = ed.lattice_translations(p, k)
            yield n, n_up, bonds, k, tr


@pytest.mark.parametrize("lat,geo,coup", CASES, ids=[c[0] for c in CASES])
def test_momentum_basis_and_hv_match_oracle(lat, geo, coup):
    """Representatives equal the oracle's bit for bit, normalisations to 1e-14; H x equals the oracle's dense
    complex matrix times x to 1e-12 of sum_j |M_ij x_j| (FP64, summation order differs)."""
    rng = np.random.default_rng(5)
    for n, n_up, bonds, k, tr in _sectors(lat, geo, coup):
        b = bloch.bloch_basis(n, n_up, tr)
        ham = ed.Hamiltonian(n, n_up, bonds, translations=tr)
        try:
            assert ham.dim == len(b["reps"]), k
            if ham.dim == 0:
                continue
            st, nm = ham.momentum_basis()
            assert np.array_equal(st, np.array(b["reps"], np.uint32)), k
            assert np.allclose(nm, b["norm"], rtol=1e-14, atol=0), k
            M = bloch.hamiltonian(n, bonds, b)
            x = rng.normal(size=ham.dim) + 1j * rng.normal(size=ham.dim)
            y = ham.apply(x)
            bound = 1e-12 * (np.abs(M) @ np.abs(x)) + 1e-14
            assert np.all(np.abs(y - M @ x) <= bound), k
        finally:
            ham.close()


@pytest.mark.parametrize("lat,geo,coup", CASES[:4], ids=[c[0] for c in CASES[:4]])
def test_momentum_lanczos_eigenvalues_match_dense(lat, geo, coup):
    """aed_solve in every momentum sector: the lowest eigenvalues of the oracle's dense matrix (1e-10), and
    the lowest over all momenta equals the Sz sector's ground state from the real path."""
    n, bonds = _bonds(lat, geo, coup)
    lows = []
    for n_, n_up, bonds_, k, tr in _sectors(lat, geo, coup, n_ups=(n // 2,)):
        b = bloch.bloch_basis(n, n_up, tr)
        ham = ed.Hamiltonian(n, n_up, bonds, translations=tr)
        try:
            if ham.dim == 0:
                continue
            ev = np.linalg.eigvalsh(bloch.hamiltonian(n, bonds, b))
            nev = min(2, ham.dim)
            r = ham.solve(nev=nev, seed=3)
            assert r["converged"]
            got = r["evals"][:nev]
            # a sector with a repeated lowest value reports it once (distinct values, like the reference)
            distinct = [ev[0]] + [v for v in ev[1:] if v - ev[0] > 1e-8][:1]
            assert np.allclose(got[:len(distinct)], distinct[:len(got)], atol=1e-10), (k, got, ev[:3])
            lows.append(got[0])
        finally:
            ham.close()
    real = ed.Hamiltonian(n, n // 2, bonds)
    e0 = real.solve(nev=1, seed=1)["evals"][0]
    real.close()
    assert abs(min(lows) - e0) < 1e-10


def test_momentum_one_state_and_empty_sectors():
    """The fully polarised sector of an 8-site chain: k = 0 holds its one state (energy L/4 J), the other
    momenta are empty."""
    lat, geo = "chain lattice", {"L": 8}
    n, bonds = _bonds(lat, geo, {0: (1.0, 1.0)})
    p = _params(lat, geo)
    dims = []
    for k in ed.lattice_momenta(p):
        ham = ed.Hamiltonian(n, n, bonds, translations=ed.lattice_translations(p, k))
        dims.append(ham.dim)
        r = ham.solve(nev=1)
        if ham.dim == 1:
            assert abs(r["evals"][0] - 2.0) < 1e-14
        else:
            assert len(r["evals"]) == 0
        ham.close()
    assert dims == [1] + [0] * 7


def test_momentum_set_couplings_and_eigenvectors():
    """New couplings on a momentum handle, then Ritz vectors: eigenvalues as the oracle's dense matrix,
    residuals |H psi - lambda psi| small, psi normalised (complex vectors)."""
    lat, geo = "nnn chain lattice", {"L": 12}
    p = _params(lat, geo)
    k = ed.lattice_momenta(p)[3]
    tr = ed.lattice_translations(p, k)
    n, b1 = _bonds(lat, geo, {0: (1.0, 1.0), 1: (0.2, 0.2)})
    _, b2 = _bonds(lat, geo, {0: (1.0, 1.0), 1: (0.35, 0.35)})
    ham = ed.Hamiltonian(n, n // 2, b1, translations=tr)
    ham.set_couplings(b2)
    r = ham.solve(nev=2, seed=4)
    ev = np.linalg.eigvalsh(bloch.hamiltonian(n, b2, bloch.bloch_basis(n, n // 2, tr)))
    assert np.allclose(r["evals"][:2], ev[:2], atol=1e-10)
    vecs, evals, res = ham.eigenvectors(k=2, seed=4)
    assert np.allclose(evals, r["evals"][:2], atol=0, rtol=0)
    for v, lam, rs in zip(vecs, evals, res):
        psi = v.download()
        assert psi.dtype == np.complex128 and psi.size == ham.dim
        assert abs(np.linalg.norm(psi) - 1) < 1e-12
        assert rs < 1e-6
    ham.close()


def test_sparsediag_loops_over_momenta():
    """sparsediag.run on a periodic chain with translation symmetry on: one sector per (Sz, k) with
    non-zero dimension, momentum innermost and labelled by write_vector(k); the ground state and gap equal
    those of the run without translation symmetry."""
    p = {"MODEL": "spin", "LATTICE": "chain lattice", "L": 8, "CONSERVED_QUANTUMNUMBERS": "Sz",
         "NUMBER_EIGENVALUES": 2}
    res = sparsediag.run(p)
    ref = sparsediag.run(dict(p, TRANSLATION_SYMMETRY="false"))
    labels = [tuple(s["quantumnumbers"]) for s in res["sectors"]]
    ks = ed.lattice_momenta(p)
    exp = []
    for m2 in range(-8, 9, 2):
        sz = sparsediag.half_integer_text(__import__("fractions").Fraction(m2, 2))
        n_up = 4 + m2 // 2
        for k in ks:
            b = bloch.bloch_basis(8, n_up, bloch.translations("chain lattice", {"L": 8}, k))
            if b["reps"]:
                exp.append((("Sz", sz), ("TOTAL_MOMENTUM", bloch.momentum_label(k))))
    assert labels == exp
    assert abs(res["ground_state_energy"] - ref["ground_state_energy"]) < 1e-10
    assert abs(res["energy_gap"] - ref["energy_gap"]) < 1e-9


def test_sparsediag_sectors_at_once_give_the_same_results():
    """sparsediag.run(workers=4) solves four sectors at a time on their own handles: every sector's
    energies, dimension and iteration count, and their order, equal the one-by-one loop's (momentum
    sectors of a chain, and the plain Sz loop of a ladder)."""
    for p in ({"MODEL": "spin", "LATTICE": "chain lattice", "L": 12, "CONSERVED_QUANTUMNUMBERS": "Sz",
               "NUMBER_EIGENVALUES": 2},
              {"MODEL": "spin", "LATTICE": "ladder", "L": 6, "J0": 1.0, "J1": 0.7, "CONSERVED_QUANTUMNUMBERS": "Sz",
               "NUMBER_EIGENVALUES": 2, "TRANSLATION_SYMMETRY": "false"}):
        one = sparsediag.run(p)
        many = sparsediag.run(p, workers=4)
        assert len(one["sectors"]) == len(many["sectors"]) > 4
        for a, b in zip(one["sectors"], many["sectors"]):
            assert a["quantumnumbers"] == b["quantumnumbers"]
            assert a["dimension"] == b["dimension"] and a["iterations"] == b["iterations"]
            assert np.array_equal(a["energies"], b["energies"])
        assert one["ground_state_energy"] == many["ground_state_energy"]


def test_momentum_rejects_couplings_that_break_translations():
    lat, geo = "chain lattice", {"L": 8}
    n, bonds = _bonds(lat, geo, {0: (1.0, 1.0)})
    bonds[3] = (bonds[3][0], bonds[3][1], 1.5, 1.5, 0.0)
    tr = ed.lattice_translations(_params(lat, geo), (0.0,))
    with pytest.raises(ed.AEDError, match="invariant"):
        ed.Hamiltonian(n, n // 2, bonds, translations=tr)


def test_momentum_set_couplings_keeps_translation_invariance():
    lat, geo = "chain lattice", {"L": 8}
    n, bonds = _bonds(lat, geo, {0: (1.0, 1.0)})
    ham = ed.Hamiltonian(n, n // 2, bonds, translations=ed.lattice_translations(_params(lat, geo), (0.0,)))
    bad = list(bonds)
    bad[2] = (bad[2][0], bad[2][1], 2.0, 2.0, 0.0)
    with pytest.raises(ed.AEDError, match="invariant"):
        ham.set_couplings(bad)
    ham.close()
