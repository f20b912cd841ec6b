"""Spin-S sectors (local_S = 1/2 .. 2) on the GPU against the oracle's Kronecker-product restatement."""

import numpy as np
import pytest
import scipy.sparse.linalg as sla

import alps_b200 as ed
from alps_b200 import sparsediag
from oracle import lattice
from oracle import spin as ospin

pytestmark = pytest.mark.gpu


def _chain(L, jz=1.0, jxy=1.0, k=0.0):
    return [(i, (i + 1) % L, jz, jxy, k) for i in range(L)]


CASES = [(2, 8, "chain"), (2, 4, "square22"), (3, 6, "chain"), (4, 5, "chain"), (1, 10, "chain")]


@pytest.mark.parametrize("two_s,n,kind", CASES, ids=[f"2S={c[0]}-{c[2]}{c[1]}" for c in CASES])
def test_spin_s_basis_and_hv_match_oracle(two_s, n, kind):
    """States in the reference's basis order, H x equal to the oracle's sparse H x (1e-12 of sum |H_ij x_j|),
    random couplings with biquadratic terms, random fields and single-ion anisotropy."""
    rng = np.random.default_rng(two_s * 100 + n)
    if kind == "chain":
        graph = [(i, (i + 1) % n) for i in range(n)]
    else:
        _, _, g = lattice.lattice_graph("square lattice", {"L": 2})
        graph = [(s, t) for s, t, _ in g]
    bonds = [(s, t, *rng.uniform(0.5, 1.5, 2), rng.uniform(-0.3, 0.3)) for s, t in graph]
    h = rng.uniform(-0.3, 0.3, n)
    dd = rng.uniform(-0.5, 0.5, n)
    for T in sorted({n * two_s // 2, n * two_s // 2 - 1}):
        ham = ed.Hamiltonian(n, T, bonds, site_h=h, site_d=dd, two_s=two_s, generic=True)
        ref_states = ospin.packed_states(n, two_s, T)
        assert ham.dim == len(ref_states)
        assert np.array_equal(ham.basis(), ref_states)
        H = ospin.hamiltonian(n, two_s, bonds, h, dd, digit_sum=T)
        x = rng.normal(size=ham.dim)
        y = ham.apply(x)
        bound = 1e-12 * (abs(H) @ np.abs(x)) + 1e-14
        assert np.all(np.abs(y - H @ x) <= bound)
        r = ham.solve(nev=2, seed=3)
        ev = np.linalg.eigvalsh(H.toarray()) if ham.dim < 3000 else sla.eigsh(H, k=4, which="SA")[0]
        ev = np.sort(ev)
        distinct = [ev[0]] + [v for v in ev[1:] if v - ev[0] > 1e-8][:1]
        assert np.allclose(r["evals"][:len(distinct)], distinct[:len(r["evals"])], atol=1e-10)
        ham.close()


def test_spin_half_through_the_spin_s_engine_matches_the_bit_exact_engine():
    rng = np.random.default_rng(4)
    n = 12
    bonds = [(i, (i + 1) % n, 1.0, 1.0, 0.0) for i in range(n)] + [(i, (i + 2) % n, 0.4, 0.4, 0.0) for i in range(n)]
    h = rng.uniform(-0.2, 0.2, n)
    a = ed.Hamiltonian(n, 6, bonds, site_h=h)
    b = ed.Hamiltonian(n, 6, bonds, site_h=h, generic=True)
    assert np.array_equal(a.basis().astype(np.uint64), b.basis())
    x = rng.normal(size=a.dim)
    assert np.allclose(a.apply(x), b.apply(x), rtol=1e-13, atol=1e-13)
    assert np.allclose(a.solve(nev=2, seed=1)["evals"], b.solve(nev=2, seed=1)["evals"], atol=1e-11)
    a.close()
    b.close()


def test_aklt_chain_closed_form():
    """S=1 chain with J = 1, K = 1/3 (the AKLT point, periodic L = 10): ground-state energy -2L/3 exactly,
    spin-1 dimer: S.S levels -2, -1, 1."""
    L = 10
    ham = ed.Hamiltonian(L, L, _chain(L, 1.0, 1.0, 1.0 / 3.0), two_s=2)
    assert abs(ham.solve(nev=1, seed=2)["evals"][0] + 2 * L / 3) < 1e-10
    ham.close()
    levels = []
    for T in (0, 1, 2):  # Sz_total = -2, -1, 0 of two spin-1 sites
        d = ed.Hamiltonian(2, T, [(0, 1, 1.0, 1.0, 0.0)], two_s=2)
        levels += list(d.solve(nev=3, seed=1)["evals"])
        d.close()
    assert np.allclose(sorted(set(np.round(levels, 12))), [-2.0, -1.0, 1.0])


def test_sparsediag_spin_one_sector_loop():
    """local_S = 1 in the parameters: sectors Sz_total = -L .. L, each against the oracle's spectrum."""
    p = {"MODEL": "spin", "LATTICE": "chain lattice", "L": 6, "J": 1, "D": 0.3, "local_S": 1,
         "CONSERVED_QUANTUMNUMBERS": "Sz", "TRANSLATION_SYMMETRY": "false", "NUMBER_EIGENVALUES": 1}
    res = sparsediag.run(p)
    labels = [s["quantumnumbers"][0][1] for s in res["sectors"]]
    assert labels == [str(k) for k in range(-6, 7)]
    for s, T in zip(res["sectors"], range(0, 13)):
        H = ospin.hamiltonian(6, 2, _chain(6), None, [0.3] * 6, digit_sum=T)
        e0 = np.linalg.eigvalsh(H.toarray())[0]
        assert abs(s["energies"][0] - e0) < 1e-10


def test_spin_s_set_couplings():
    """New couplings on a spin-1 handle: the eigenvalues follow (oracle dense spectrum)."""
    n = 8
    ham = ed.Hamiltonian(n, n, _chain(n), two_s=2)
    ham.set_couplings(_chain(n, 1.0, 0.5, 0.2))
    H = ospin.hamiltonian(n, 2, _chain(n, 1.0, 0.5, 0.2), digit_sum=n)
    e0 = np.linalg.eigvalsh(H.toarray())[0]
    assert abs(ham.solve(nev=1, seed=1)["evals"][0] - e0) < 1e-10
    ham.close()


def test_spin_s_set_couplings_through_every_apply_form():
    """One spin-3/2 handle (8 sites: bonds inside the lo word, inside the hi word and across) through
    new couplings that change the apply's form: Heisenberg (two off-diagonal slots, lo table), with a
    biquadratic term (three slots, no lo table), one class per bond (16 classes, more than 8: per-bond
    form), and Heisenberg again with next-nearest bonds (a longer lo table); H x equals the oracle's
    each time (1e-12 of sum |H_ij x_j|)."""
    n, two_s, T = 8, 3, 12
    rng = np.random.default_rng(31)
    nnn = [(i, (i + 2) % n, 0.4, 0.3, 0.0) for i in range(n)]
    forms = [_chain(n, 1.0, 0.8), _chain(n, 1.0, 1.0, 0.25),
             [(s, t, *rng.uniform(0.5, 1.5, 2), rng.uniform(-0.3, 0.3)) for s, t, *_ in _chain(n) + nnn],
             _chain(n) + nnn]
    ham = ed.Hamiltonian(n, T, forms[0], two_s=two_s)
    try:
        for bonds in forms:
            ham.set_couplings(bonds)
            H = ospin.hamiltonian(n, two_s, bonds, digit_sum=T)
            x = rng.normal(size=ham.dim)
            y = ham.apply(x)
            assert np.all(np.abs(y - H @ x) <= 1e-12 * (abs(H) @ np.abs(x)) + 1e-14)
    finally:
        ham.close()


@pytest.mark.parametrize("two_s,n", [(4, 7), (3, 8)], ids=["2S=4-chain7", "2S=3-chain8"])
def test_spin_s_lo_table_with_site_terms(two_s, n):
    """Spin 2 and spin 3/2 with nearest and next-nearest Heisenberg bonds (two coupling classes, no
    biquadratic term: two off-diagonal slots, so the apply reads the lo table), fields and single-ion
    anisotropy on every site: H x equals the oracle's (1e-12 of sum |H_ij x_j|) in two Sz sectors."""
    rng = np.random.default_rng(two_s * 31 + n)
    bonds = _chain(n, 1.0, 0.9) + [(i, (i + 2) % n, 0.35, 0.3, 0.0) for i in range(n)]
    h = rng.uniform(-0.3, 0.3, n)
    dd = rng.uniform(-0.5, 0.5, n)
    for T in (n * two_s // 2, n * two_s // 2 - 1):
        ham = ed.Hamiltonian(n, T, bonds, site_h=h, site_d=dd, two_s=two_s)
        H = ospin.hamiltonian(n, two_s, bonds, h, dd, digit_sum=T)
        x = rng.normal(size=ham.dim)
        y = ham.apply(x)
        assert np.all(np.abs(y - H @ x) <= 1e-12 * (abs(H) @ np.abs(x)) + 1e-14)
        ham.close()


SPIN_MEAS = {
    "MEASURE_AVERAGE[Magnetization]": "Sz",
    "MEASURE_LOCAL[Local magnetization]": "Sz",
    "MEASURE_CORRELATIONS[Diagonal spin correlations]": "Sz",
    "MEASURE_CORRELATIONS[Offdiagonal spin correlations]": "Splus:Sminus",
    "MEASURE_CORRELATIONS[Reverse offdiagonal]": "Sminus:Splus",
    "MEASURE_STRUCTURE_FACTOR[Structure Factor S]": "Sz",
    "MEASURE_STRUCTURE_FACTOR[Structure Factor mp]": "Sminus:Splus",
}


@pytest.mark.parametrize("two_s,n", [(2, 8), (3, 6), (4, 5)])
def test_spin_s_expectation_matches_oracle(two_s, n):
    """aed_expectation on a spin-S handle: <Sz_i>, <Sz_i Sz_j>, <S+_i S-_j> for every site pair of a random
    vector equal the oracle's Kronecker-product operators (1e-12 relative)."""
    from alps_b200 import measure
    rng = np.random.default_rng(two_s * 7 + n)
    T = n * two_s // 2 - 1
    ham = ed.Hamiltonian(n, T, _chain(n), two_s=two_s)
    psi = rng.normal(size=ham.dim)
    v = ham.new_vector().upload(psi)
    si = np.repeat(np.arange(n), n)
    sj = np.tile(np.arange(n), n)
    got_z = measure.expectation(ham, v, measure.OBS_SZ, np.arange(n))
    got_zz = measure.expectation(ham, v, measure.OBS_SZSZ, si, sj)
    got_pm = measure.expectation(ham, v, measure.OBS_SPSM, si, sj)
    scale = float(psi @ psi) * (two_s / 2.0 + 1) ** 2
    for i in range(n):
        ref = ospin.pair_expectation(n, two_s, T, psi, [("Sz", i)])
        assert abs(got_z[i] - ref) <= 1e-12 * scale
    for p, (i, j) in enumerate(zip(si, sj)):
        ref = ospin.pair_expectation(n, two_s, T, psi, [("Sz", i), ("Sz", j)])
        assert abs(got_zz[p] - ref) <= 1e-12 * scale, (i, j)
        ref = ospin.pair_expectation(n, two_s, T, psi, [("Splus", i), ("Sminus", j)])
        assert abs(got_pm[p] - ref) <= 1e-12 * scale, (i, j)
    v.free()
    ham.close()


@pytest.mark.parametrize("lat,geo,two_s", [("ladder", {"L": 4}, 2), ("chain lattice", {"L": 6}, 3),
                                           ("open chain lattice", {"L": 5}, 4)])
def test_spin_s_measurements_match_oracle(lat, geo, two_s):
    """MEASURE_* quantities of the ground state of a spin-S sector (random couplings and fields: no
    degeneracy) equal the oracle's on the dense eigenvector (1e-8: Ritz vectors to |H psi - E psi| ~ 1e-9)."""
    from alps_b200 import measure
    from oracle import measure as omeasure
    rng = np.random.default_rng(two_s + 31)
    n, _, graph = lattice.lattice_graph(lat, geo)
    bonds = [(s, t, float(j), float(j), 0.0) for (s, t, _), j in zip(graph, rng.uniform(0.7, 1.3, len(graph)))]
    h = rng.uniform(-0.2, 0.2, n)
    params = dict(geo, LATTICE=lat, **SPIN_MEAS)
    T = n * two_s // 2
    ham = ed.Hamiltonian(n, T, bonds, site_h=h, two_s=two_s)
    ham.solve(nev=1, seed=2)
    vecs, ev, _ = ham.eigenvectors(k=1, seed=2)
    H = ospin.hamiltonian(n, two_s, bonds, h, None, digit_sum=T).toarray()
    w, Z = np.linalg.eigh(H)
    assert abs(w[0] - ev[0]) < 1e-9 and w[1] - w[0] > 1e-6
    got = measure.measure(ham, vecs[0], params)
    ref = omeasure.measure(ham.basis(), Z[:, 0], params, two_s)
    for key in ref:
        for name in ref[key]:
            a, b = np.asarray(got[key][name], float), np.asarray(ref[key][name], float)
            assert a.shape == b.shape, (key, name)
            assert np.allclose(a, b, atol=1e-8), (key, name, a, b)
    vecs[0].free()
    ham.close()


def test_sparsediag_spin_one_measurements():
    """local_S = 1 Heisenberg ring through sparsediag.run: zero magnetization at Sz_total = 0 and
    <S_0 . S_1> = E0 / L (Sz Sz plus half of S+ S- and S- S+ at distance 1)."""
    L = 6
    p = {"MODEL": "spin", "LATTICE": "chain lattice", "L": L, "J": 1, "local_S": 1, "CONSERVED_QUANTUMNUMBERS": "Sz",
         "Sz_total": 0, "NUMBER_EIGENVALUES": 1, "TRANSLATION_SYMMETRY": "false", **SPIN_MEAS}
    res = sparsediag.run(p)
    m = res["sectors"][0]["measurements"][0]
    assert abs(m["average"]["Magnetization"]) < 1e-12
    c = m["correlations"]
    d1 = c["Diagonal spin correlations"][1] + 0.5 * (c["Offdiagonal spin correlations"][1] +
                                                      c["Reverse offdiagonal"][1])
    assert abs(d1 - res["ground_state_energy"] / L) < 1e-9
    # on one site S.S = S(S+1) = 2: Sz^2 + (S+ S- + S- S+) / 2
    d0 = c["Diagonal spin correlations"][0] + 0.5 * (c["Offdiagonal spin correlations"][0] +
                                                      c["Reverse offdiagonal"][0])
    assert abs(d0 - 2.0) < 1e-9


SPIN_MOM_CASES = [(2, "chain lattice", {"L": 6}), (3, "chain lattice", {"L": 5}), (4, "chain lattice", {"L": 4}),
                  (2, "square lattice", {"L": 2, "W": 3})]


@pytest.mark.parametrize("two_s,lat,geo", SPIN_MOM_CASES, ids=[f"2S={c[0]}-{c[1]}" for c in SPIN_MOM_CASES])
def test_spin_s_momentum_sectors_match_oracle(two_s, lat, geo):
    """Spin-S momentum sectors (aed_create_spin_momentum): representatives equal the oracle's Bloch basis
    over packed digits, normalisations to 1e-14, H x equal to the oracle's complex matrix (built from the
    sector's Kronecker-product H) to 1e-12 of sum |M_ij x_j|, the lowest eigenvalues to 1e-10, and the
    dimensions over all momenta add up to the Sz sector's."""
    from oracle import bloch
    rng = np.random.default_rng(two_s * 13 + len(geo))
    n, _, graph = lattice.lattice_graph(lat, geo)
    bonds = [(s, t, 1.0, 0.9, 0.15) for s, t, _ in graph]
    h, dd = [0.1] * n, [0.25] * n
    bits = two_s.bit_length()
    p = dict(geo, MODEL="spin", LATTICE=lat, CONSERVED_QUANTUMNUMBERS="Sz")
    for T in (n * two_s // 2, n * two_s // 2 - 1):
        H = ospin.hamiltonian(n, two_s, bonds, h, dd, digit_sum=T)
        states = ospin.packed_states(n, two_s, T)
        total = 0
        for k in ed.lattice_momenta(p):
            tr = ed.lattice_translations(p, k)
            b = bloch.bloch_basis_of(states, n, tr, lambda s, mp: bloch.translate_digits(s, mp, n, bits))
            ham = ed.Hamiltonian(n, T, bonds, site_h=h, site_d=dd, translations=tr, two_s=two_s)
            try:
                assert ham.dim == len(b["reps"]), k
                total += ham.dim
                if ham.dim == 0:
                    continue
                st, nm = ham.momentum_basis()
                assert np.array_equal(st, np.array(b["reps"], np.uint64)), k
                assert np.allclose(nm, b["norm"], rtol=1e-14, atol=0), k
                M = bloch.hamiltonian_from_sector(H, states, b)
                x = rng.normal(size=ham.dim) + 1j * rng.normal(size=ham.dim)
                y = ham.apply(x)
                bound = 1e-12 * (np.abs(M) @ np.abs(x)) + 1e-14
                assert np.all(np.abs(y - M @ x) <= bound), k
                ev = np.sort(np.linalg.eigvals(M).real)
                r = ham.solve(nev=1, seed=3)
                assert r["converged"] and abs(r["evals"][0] - ev[0]) < 1e-10, k
            finally:
                ham.close()
        assert total == len(states)


def test_sparsediag_spin_one_momentum_loop():
    """local_S = 1 with the reference's default TRANSLATION_SYMMETRY: every (Sz, TOTAL_MOMENTUM) sector, whose
    lowest values over all momenta equal each Sz sector's ground state without translation symmetry."""
    L = 6
    p = {"MODEL": "spin", "LATTICE": "chain lattice", "L": L, "J": 1, "D": 0.2, "local_S": 1,
         "CONSERVED_QUANTUMNUMBERS": "Sz", "NUMBER_EIGENVALUES": 1}
    res = sparsediag.run(p)
    plain = sparsediag.run(dict(p, TRANSLATION_SYMMETRY="false"))
    names = {tuple(q[0] for q in s["quantumnumbers"]) for s in res["sectors"]}
    assert names == {("Sz", "TOTAL_MOMENTUM")}
    for s0 in plain["sectors"]:
        sz = s0["quantumnumbers"][0][1]
        lows = [s["energies"][0] for s in res["sectors"] if s["quantumnumbers"][0][1] == sz]
        assert abs(min(lows) - s0["energies"][0]) < 1e-10, sz
    assert abs(res["ground_state_energy"] - plain["ground_state_energy"]) < 1e-10


def test_spin_s_momentum_sector_measurements():
    """Spin-1 ring with translation symmetry: the sector of the (non-degenerate) Sz=0 ground state reports
    the class-averaged correlations, the average and the structure factors the oracle computes on the dense
    ground state (1e-8)."""
    from oracle import measure as omeasure
    L = 6
    meas = {k: v for k, v in SPIN_MEAS.items() if "LOCAL" not in k}
    p = {"MODEL": "spin", "LATTICE": "chain lattice", "L": L, "J": 1, "D": 0.2, "local_S": 1,
         "CONSERVED_QUANTUMNUMBERS": "Sz", "Sz_total": 0, "NUMBER_EIGENVALUES": 1, **meas}
    res = sparsediag.run(p)
    best = min(res["sectors"], key=lambda s: s["energies"][0])
    got = best["measurements"][0]
    H = ospin.hamiltonian(L, 2, _chain(L), None, [0.2] * L, digit_sum=L)
    w, Z = np.linalg.eigh(H.toarray())
    assert abs(w[0] - best["energies"][0]) < 1e-9 and w[1] - w[0] > 1e-6
    ref = omeasure.measure_translation_invariant(ospin.packed_states(L, 2, L), Z[:, 0], p, 2)
    assert got["local"] == {}
    for key in ref:
        for name in ref[key]:
            a, b = np.asarray(got[key][name], float), np.asarray(ref[key][name], float)
            assert a.shape == b.shape, (key, name)
            assert np.allclose(a, b, atol=1e-8), (key, name, a, b)


def test_basis_state_of_every_kind_of_handle():
    """aed_basis_state: row idx of a spin-1/2 Sz sector, a spin-1/2 momentum sector, a spin-S Sz sector and a
    spin-S momentum sector equals the handle's basis listing at that row; out-of-range rows are refused."""
    p = {"MODEL": "spin", "LATTICE": "chain lattice", "L": 6, "CONSERVED_QUANTUMNUMBERS": "Sz"}
    k = ed.lattice_momenta(p)[1]
    tr = ed.lattice_translations(p, k)
    bonds = _chain(6)
    hams = [ed.Hamiltonian(6, 3, bonds), ed.Hamiltonian(6, 3, bonds, translations=tr),
            ed.Hamiltonian(6, 6, bonds, two_s=2), ed.Hamiltonian(6, 6, bonds, translations=tr, two_s=2)]
    for ham in hams:
        listing = ham.momentum_basis()[0] if ham.momentum else ham.basis()
        for idx in (0, ham.dim // 2, ham.dim - 1):
            assert ham.state(idx) == int(listing[idx])
        with pytest.raises(ed.AEDError):
            ham.state(ham.dim)
        ham.close()


def test_parameter_file_with_odd_spin_one_chain():
    """A parameter file of two spin-1 chain tasks (L = 5 and 4, every Sz sector) through sparsediag.run_list: the
    odd chain loops over Sz_total = -5 .. 5, and every sector's lowest value equals the oracle's dense spectrum."""
    txt = ('MODEL="spin"; LATTICE="chain lattice"; CONSERVED_QUANTUMNUMBERS="Sz"; local_S=1; J=1;\n'
           'TRANSLATION_SYMMETRY=false; NUMBER_EIGENVALUES=1\n{ L=5 }\n{ L=4; D=0.3 }\n')
    out = sparsediag.run_list(txt)
    assert [p["L"] for p, _ in out] == ["5", "4"]
    for (p, res), dd in zip(out, (0.0, 0.3)):
        L = int(p["L"])
        labels = [s["quantumnumbers"][0][1] for s in res["sectors"]]
        assert labels == [str(k) for k in range(-L, L + 1)]
        for s, T in zip(res["sectors"], range(0, 2 * L + 1)):
            H = ospin.hamiltonian(L, 2, _chain(L), None, [dd] * L, digit_sum=T)
            assert abs(s["energies"][0] - np.linalg.eigvalsh(H.toarray())[0]) < 1e-10
