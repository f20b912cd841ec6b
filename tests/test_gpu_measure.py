"""Eigenvector measurements (MEASURE_* of sparsediag) on the GPU against the oracle's restatement."""

import numpy as np
import pytest

import alps_b200 as ed
import oracle
from alps_b200 import measure, sparsediag
from oracle import lattice
from oracle import measure as omeasure

pytestmark = pytest.mark.gpu

MEAS = {
    "MEASURE_AVERAGE[Magnetization]": "Sz",
    "MEASURE_LOCAL[Local magnetization]": "Sz",
    "MEASURE_CORRELATIONS[Diagonal spin correlations]": "Sz",
    "MEASURE_CORRELATIONS[Offdiagonal spin correlations]": "Splus:Sminus",
    "MEASURE_CORRELATIONS[Reverse offdiagonal]": "Sminus:Splus",
    "MEASURE_CORRELATIONS[Mixed]": "Sz:Splus",
    "MEASURE_STRUCTURE_FACTOR[Structure Factor S]": "Sz",
    "MEASURE_STRUCTURE_FACTOR[Structure Factor pm]": "Splus:Sminus",
}

CASES = [("open chain lattice", {"L": 10}), ("chain lattice", {"L": 10}), ("square lattice", {"L": 4, "W": 3}),
         ("ladder", {"L": 5}), ("anisotropic square lattice", {"L": 3, "W": 3})]


def _dense(n, n_up, bonds, h):
    st = oracle.basis(n, n_up)
    M = oracle.Matrix(n, n_up, bonds, site_h=h)
    D = len(st)
    A = np.zeros((D, D))
    for j in range(D):
        e = np.zeros(D)
        e[j] = 1.0
        A[:, j] = M.mult(e)
    return st, A


def _close(got, ref, tol):
    for key in ref:
        for name in ref[key]:
            a, b = np.asarray(got[key][name], float), np.asarray(ref[key][name], float)
            assert a.shape == b.shape, (key, name)
            assert np.allclose(a, b, atol=tol), (key, name, a, b)


@pytest.mark.parametrize("lat,geo", CASES, ids=[c[0] for c in CASES])
def test_measurements_match_oracle(lat, geo):
    """Averages, local values, correlations per distance class and structure factors of the two lowest
    eigenvectors (random couplings and fields: no degeneracy) equal the oracle's on dense eigenvectors
    (1e-8: Ritz vectors to |H psi - E psi| ~ 1e-9)."""
    rng = np.random.default_rng(11)
    n, _, graph = lattice.lattice_graph(lat, geo)
    bonds = [(s, t, float(j), float(j), 0.0) for (s, t, _), j in zip(graph, rng.uniform(0.7, 1.3, len(graph)))]
    h = rng.uniform(-0.2, 0.2, n)
    params = dict(geo, LATTICE=lat, **MEAS)
    g = measure.Geometry(params)
    for n_up in (n // 2, n // 2 - 1):
        ham = ed.Hamiltonian(n, n_up, bonds, site_h=h)
        r = ham.solve(nev=2, seed=2)
        vecs, ev, _ = ham.eigenvectors(k=2, seed=2)
        st, A = _dense(n, n_up, bonds, h)
        w, Z = np.linalg.eigh(A)
        for v, lam in zip(vecs, ev):
            k = int(np.argmin(np.abs(w - lam)))
            assert abs(w[k] - lam) < 1e-9
            assert min(abs(w[kk] - lam) for kk in range(len(w)) if kk != k) > 1e-6  # non-degenerate
            got = measure.measure(ham, v, params, g)
            ref = omeasure.measure(st, Z[:, k], params)
            _close(got, ref, 1e-8)
        ham.close()


def test_sparsediag_attaches_measurements():
    p = {"MODEL": "spin", "LATTICE": "chain lattice", "L": 8, "J": 1, "CONSERVED_QUANTUMNUMBERS": "Sz", "Sz_total": 0,
         "NUMBER_EIGENVALUES": 1, "TRANSLATION_SYMMETRY": "false", **MEAS}
    res = sparsediag.run(p)
    m = res["sectors"][0]["measurements"][0]
    assert abs(m["average"]["Magnetization"]) < 1e-12
    # Heisenberg ring ground state: <S_0 . S_1> = E0 / L per bond
    e0 = res["ground_state_energy"]
    d1 = m["correlations"]["Diagonal spin correlations"][1] + m["correlations"]["Offdiagonal spin correlations"][1]
    assert abs(d1 - e0 / 8) < 1e-9


def test_zero_coupling_stops_at_the_invariant_space():
    """J = 0 (the spin model's default): H = 0, beta_0 = 0 exactly; the recurrence stops with the exact value 0
    instead of dividing by zero."""
    p = {"MODEL": "spin", "LATTICE": "chain lattice", "L": 8, "CONSERVED_QUANTUMNUMBERS": "Sz", "Sz_total": 0,
         "TRANSLATION_SYMMETRY": "false"}
    ham = ed.Hamiltonian.from_parameters(p)
    r = ham.solve(nev=2, seed=1)
    assert r["converged"] and r["iterations"] == 1
    assert list(r["evals"]) == [0.0]
    vecs, ev, res = ham.eigenvectors(k=1, seed=1)
    assert ev[0] == 0.0 and res[0] == 0.0
    ham.close()


@pytest.mark.parametrize("lat,geo,couplings", [("nnn chain lattice", {"L": 10}, {"J": 1, "J1": 0.3}),
                                               ("square lattice", {"L": 4, "W": 3}, {"J": 1})])
def test_momentum_sector_measurements(lat, geo, couplings):
    """With translation symmetry on, the sector holding the ground state reports the class-averaged
    correlations, the average and the structure factors of the (non-degenerate) Sz=0 ground state,
    computed by the oracle on the dense ground state (1e-8)."""
    p = dict(geo, MODEL="spin", LATTICE=lat, CONSERVED_QUANTUMNUMBERS="Sz", Sz_total=0, NUMBER_EIGENVALUES=1,
             **couplings, **{k: v for k, v in MEAS.items() if "LOCAL" not in k})
    res = sparsediag.run(p)
    best = min(res["sectors"], key=lambda s: s["energies"][0])
    got = best["measurements"][0]
    n, n_up, bonds = lattice.spin_model(dict(p, TRANSLATION_SYMMETRY="false"))
    st, A = _dense(n, n_up, bonds, None)
    w, Z = np.linalg.eigh(A)
    assert abs(w[0] - best["energies"][0]) < 1e-9 and w[1] - w[0] > 1e-6
    ref = omeasure.measure_translation_invariant(st, Z[:, 0], p)
    assert got["local"] == {}
    _close(got, ref, 1e-8)
