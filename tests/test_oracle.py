"""The oracle pinned against the reference's own golden outputs, LAPACK and closed forms (CPU)."""

import json
import os
import re

import numpy as np
import pytest

import oracle
from oracle import bloch, lattice

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def gold(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def sz_rows_to_bits(rows):
    """[+1/-1 per site] -> bit strings, site 0 most significant (up = 1)."""
    n = len(rows[0])
    out = []
    for r in rows:
        v = 0
        for s, sz in enumerate(r):
            if sz > 0:
                v |= 1 << (n - 1 - s)
        out.append(v)
    return np.array(out, dtype=np.uint32)


def test_basis_example10_full_space_order():
    g = gold("basis_example10.json")
    bits = sz_rows_to_bits(g["states_sz"])
    # no constraint: all 16 states, lexicographic with site 0 most significant
    assert list(bits) == list(range(16))
    # the union of the Sz sectors of the oracle, in order, is the same list
    union = np.sort(np.concatenate([oracle.basis(4, k) for k in range(5)]))
    assert list(union) == list(bits)


def test_basis_example12_sz0_order():
    g = gold("basis_example12.json")
    bits = sz_rows_to_bits(g["states_sz"])
    assert list(oracle.basis(4, 2)) == list(bits)


@pytest.mark.parametrize("N,k", [(1, 0), (5, 2), (8, 4), (12, 5), (16, 8), (10, 0), (10, 10)])
def test_basis_is_ascending_popcount_sector(N, k):
    from math import comb

    b = oracle.basis(N, k)
    assert b.size == comb(N, k)
    assert np.all(np.diff(b.astype(np.int64)) > 0)
    assert all(bin(int(v)).count("1") == k for v in b)
    # lower_bound index and "absent" -> D
    for i in [0, b.size // 2, b.size - 1]:
        assert oracle.index(b, int(b[i])) == i
    if k < N:
        absent = (1 << N) - 1
        assert oracle.index(b, absent) == b.size


def test_lattice_example5_sites():
    g = gold("lattice_example5.json")
    n, coords, _ = lattice.lattice_graph(g["params"]["LATTICE"], g["params"])
    assert n == len(g["sites"])
    for s in g["sites"]:
        assert [float(c) for c in coords[s["site"]]] == s["coords"]


def test_lattice_example6_bonds():
    g = gold("lattice_example6.json")
    _, _, bonds = lattice.lattice_graph(g["params"]["LATTICE"], g["params"])
    assert [list(b) for b in bonds] == g["bonds"]


def _eval_matrix_expr(expr, vals):
    """A matrix element of the reference's symbolic output at the given couplings (numbers, + - * /, parens)."""
    e = expr.replace(" ", "")
    for k, v in vals.items():
        e = e.replace(k, f"({float(v)!r})")
    assert re.fullmatch(r"[0-9eE.+\-*/()]*", e), expr
    return eval(e) if e else 0.0


def _nested_eval(obj, vals):
    if isinstance(obj, list):
        return [_nested_eval(o, vals) for o in obj]
    return _eval_matrix_expr(obj, vals)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_spin_bond_and_site_terms_example3_example4(seed):
    rng = np.random.default_rng(seed)
    jz, jxy, k, h, d = rng.uniform(-2, 2, 5)
    vals = {"Jz0": jz, "Jxy0": jxy, "K0": k, "h0": h, "D0": d, "Gamma0": 0.0}
    # two sites, one bond, both site terms: the reference's HSpinHalf (example4)
    g4 = np.array(_nested_eval(gold("spin_half_example4.json")["HSpinHalf"], vals), dtype=float)
    full = np.zeros((4, 4))
    for nup in range(3):
        m = oracle.Matrix(2, nup, [(0, 1, jz, jxy, k)], site_h=[h, h], site_d=[d, d])
        st = m.states()
        dm = m.dense()
        for a in range(m.D):
            for b in range(m.D):
                full[st[a], st[b]] = dm[a, b]
    # HSpinHalf rows/cols are the two-site product states in order (0,0),(0,1),(1,0),(1,1)
    # of the site-basis index, i.e. bit strings 00,01,10,11
    np.testing.assert_allclose(full, g4, rtol=0, atol=1e-13)
    # bond tensor alone (example3 HSpinBond): [is1][is2][js1][js2]
    g3 = np.array(_nested_eval(gold("spin_terms_example3.json")["HSpinBond"], vals), dtype=float)
    full_b = np.zeros((4, 4))
    for nup in range(3):
        m = oracle.Matrix(2, nup, [(0, 1, jz, jxy, k)])
        st = m.states()
        dm = m.dense()
        for a in range(m.D):
            for b in range(m.D):
                full_b[st[a], st[b]] = dm[a, b]
    for is1 in range(2):
        for is2 in range(2):
            for js1 in range(2):
                for js2 in range(2):
                    # M(i,j) with i = source (is1,is2), j = target (js1,js2)
                    assert abs(full_b[(is1 << 1) | is2, (js1 << 1) | js2] - g3[is1][is2][js1][js2]) < 1e-13


def test_stev_matches_lapack():
    from scipy.linalg import lapack

    rng = np.random.default_rng(5)
    for n in [1, 2, 3, 10, 57, 200]:
        d = rng.normal(size=n)
        e = rng.uniform(0.1, 1, size=max(n - 1, 0))
        w, zl, zf = oracle.stev(d, e, want_last=True, want_full=True)
        if n > 1:
            wl, zz, info = lapack.dstev(d.copy(), e.copy(), compute_v=1)[:3]
        else:
            wl, zz = d.copy(), np.ones((1, 1))
        np.testing.assert_allclose(w, wl, rtol=0, atol=1e-13 * max(1, np.abs(wl).max()))
        np.testing.assert_allclose(np.abs(zl), np.abs(zz[-1]), atol=1e-10)
        T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
        np.testing.assert_allclose(T @ zf, zf * w, atol=1e-11)


def test_tmatrix_rules_match_lapack_restatement():
    p = {"LATTICE": "chain lattice", "L": 14, "J": 1, "Sz_total": 0}
    N, nu, bonds = lattice.spin_model(p)
    M = oracle.Matrix(N, nu, bonds)
    r = M.lanczos(nev=4, seed=11)
    a, b = r["alpha"], r["beta"]
    for m in [2, 5, 20, len(a) // 2, len(a)]:
        t1 = oracle.tmatrix(a[:m], b[:m])
        t2 = oracle.tmatrix_lapack(a[:m], b[:m])
        assert len(t1["evals"]) == len(t2["evals"])
        np.testing.assert_allclose(t1["evals"], t2["evals"], rtol=1e-12, atol=1e-12)
        assert list(t1["mults"]) == list(t2["mults"])
        np.testing.assert_allclose(t1["errors"], t2["errors"], rtol=1e-5, atol=1e-14)


def test_closed_forms():
    eps = 1e-12
    # two-site dimer: singlet -3J/4
    m = oracle.Matrix(2, 1, [(0, 1, 1.0, 1.0, 0.0)])
    assert abs(np.linalg.eigvalsh(m.dense())[0] + 0.75) < eps
    # 4-site ring: -2J
    p = {"LATTICE": "chain lattice", "L": 4, "J": 1, "Sz_total": 0}
    N, nu, bonds = lattice.spin_model(p)
    m = oracle.Matrix(N, nu, bonds)
    assert abs(np.linalg.eigvalsh(m.dense())[0] + 2.0) < eps
    # Majumdar-Ghosh point of the J1-J2 chain (J2 = J1/2, periodic even L): -3 L / 8
    for L in (8, 10, 12):
        p = {"LATTICE": "nnn chain lattice", "L": L, "J": 1, "J1": 0.5, "Sz_total": 0}
        N, nu, bonds = lattice.spin_model(p)
        m = oracle.Matrix(N, nu, bonds)
        r = m.lanczos(nev=1, seed=3)
        assert abs(r["evals"][0] + 3 * L / 8) < 1e-11


@pytest.mark.parametrize("params,nev", [
    ({"LATTICE": "chain lattice", "L": 12, "J": 1, "Sz_total": 0}, 4),
    ({"LATTICE": "nnn chain lattice", "L": 12, "J": 1, "J1": 0.37, "Sz_total": 0}, 2),
    ({"LATTICE": "ladder", "L": 5, "J0": 1.1, "J1": 0.7, "Sz_total": 0}, 3),
    ({"LATTICE": "square lattice", "L": 3, "W": 4, "J": 1, "Sz_total": 1}, 2),
    ({"LATTICE": "open chain lattice", "L": 11, "J": 1, "Sz_total": 0.5}, 2),
])
def test_oracle_lanczos_matches_dense(params, nev):
    N, nu, bonds = lattice.spin_model(params)
    m = oracle.Matrix(N, nu, bonds)
    w = np.linalg.eigvalsh(m.dense())
    distinct = [w[0]]
    for v in w[1:]:
        if v - distinct[-1] > 1e-8:
            distinct.append(v)
    r = m.lanczos(nev=nev, seed=7)
    np.testing.assert_allclose(r["evals"], distinct[:nev], rtol=1e-12, atol=1e-12)
    assert r["fail"] == 0


def test_csr_is_symmetric_and_matches_matfree():
    p = {"LATTICE": "nnn chain lattice", "L": 12, "J": 1, "J1": 0.3, "Sz_total": 0}
    N, nu, bonds = lattice.spin_model(p)
    m = oracle.Matrix(N, nu, bonds)
    H = m.dense()
    assert np.array_equal(H, H.T)
    x = np.random.default_rng(0).normal(size=m.D)
    y1 = m.mult(x)
    y2 = oracle.hv_matfree(N, m.states(), bonds, x)
    assert np.array_equal(y1, y2)


@pytest.mark.parametrize("seed", [0, 1])
def test_row_windows_equal_the_whole_explicit_matrix(seed):
    """oracle.rows_mult (the windows the full-size GPU parity tests sample) builds the same rows as the
    whole explicit matrix, bit for bit, with site terms, biquadratic couplings and duplicate bonds."""
    n, _, raw = lattice.lattice_graph("square lattice", {"L": 4, "W": 4})
    rng = np.random.default_rng(seed)
    bonds = [(s, t, float(j), float(j) * 0.7, 0.1 * seed) for (s, t, _), j in zip(raw, rng.uniform(0.5, 1.5, len(raw)))]
    bonds.append(bonds[3])
    sh, sd = rng.normal(size=n), rng.normal(size=n)
    m = oracle.Matrix(n, 8, bonds, site_h=sh, site_d=sd)
    x = rng.normal(size=m.D)
    y = m.mult(x)
    states = oracle.basis_fast(n, 8)
    rp, col, val = m.csr()
    absrow = np.add.reduceat(np.abs(val) * np.abs(x[col]), rp[:-1])
    for r0, r1 in [(0, 1), (0, 700), (5000, 9000), (m.D - 333, m.D)]:
        yw, ya = oracle.rows_mult(n, states, bonds, x, r0, r1, site_h=sh, site_d=sd)
        assert np.array_equal(yw, y[r0:r1])
        np.testing.assert_allclose(ya, absrow[r0:r1], rtol=1e-14)


# ---------------------------------------------------------------- momentum sectors
def _bloch_cases():
    out = []
    for ex in ("13", "14", "15"):
        g = json.load(open(os.path.join(GOLD, f"bloch_example{ex}.json")))
        params = {"L": g["L"]}
        n = g["L"] if g["lattice"] == "chain lattice" else g["L"] * g["L"]
        for isec, sec in enumerate(g["sections"]):
            if sec["momentum"] is not None:  # example15 prints k
                k = sec["momentum"]
                exact = [kk for kk in bloch.translation_momenta(g["lattice"], params)
                         if np.allclose(kk, k, atol=1e-5)]
                assert len(exact) == 1
                k = exact[0]
            elif ex == "13":  # k = 2 pi m / L, m = section index
                k = (2.0 * isec * np.pi / n,)
            else:  # example14: k = (0, 0)
                k = (0.0, 0.0)
            out.append((ex, g["lattice"], params, n, k, sec))
    return out


@pytest.mark.parametrize("case", _bloch_cases(), ids=lambda c: f"ex{c[0]}-k{','.join('%.2f' % v for v in c[4])}")
def test_bloch_translations_and_basis_pinned(case):
    """Translations (phases, site maps) and the Bloch basis (representatives in order, normalisations)
    against the reference's test/model/example13-15 outputs."""
    ex, lat, params, n, k, sec = case
    tr = bloch.translations(lat, params, k)
    assert len(tr) == len(sec["translations"])
    for (phase, mp), g in zip(tr, sec["translations"]):
        assert mp == g["map"]
        assert abs(round(phase.real, 1) - g["phase"][0]) < 1e-9 and abs(round(phase.imag, 1) - g["phase"][1]) < 1e-9
    b = bloch.bloch_basis(n, None, tr)
    assert len(b["reps"]) == len(sec["states"])
    for r, nm, g in zip(b["reps"], b["norm"], sec["states"]):
        sz = [1 if (r >> (n - 1 - i)) & 1 else -1 for i in range(n)]
        assert sz == g["sz"]
        assert abs(nm - g["norm"]) <= 5e-6 * g["norm"]


def test_bloch_spectra_union_is_the_sector_spectrum():
    """The eigenvalues of all momentum sectors together are those of the Sz sector (J1-J2 chain and a
    4x3 square lattice with random couplings per bond type)."""
    cases = [("chain lattice", {"L": 10}, [(0, 1.0, 1.0), (1, 0.0, 0.0)]),
             ("nnn chain lattice", {"L": 10}, [(0, 1.0, 1.0), (1, 0.4, 0.4)]),
             ("square lattice", {"L": 4, "W": 3}, [(0, 1.0, 0.8)]),
             ("ladder", {"L": 5}, [(0, 1.0, 1.0), (1, 0.7, 0.7)])]
    for lat, params, types in cases:
        n, _, graph = lattice.lattice_graph(lat, params)
        coup = {t: (jz, jxy) for t, jz, jxy in types}
        bonds = [(s, t, coup[ty][0], coup[ty][1], 0.0) for s, t, ty in graph]
        for n_up in (n // 2, n // 2 - 1):
            full = []
            for k in bloch.translation_momenta(lat, params):
                b = bloch.bloch_basis(n, n_up, bloch.translations(lat, params, k))
                M = bloch.hamiltonian(n, bonds, b)
                assert np.allclose(M, M.conj().T, atol=1e-12)
                full += list(np.linalg.eigvalsh(M))
            ref = np.linalg.eigvalsh(_dense_real(n, n_up, bonds, oracle.basis(n, n_up)))
            assert np.allclose(np.sort(full), ref, atol=1e-10), lat


def _dense_real(n, n_up, bonds, st):
    M = oracle.Matrix(n, n_up, bonds)
    D = len(st)
    out = np.zeros((D, D))
    for j in range(D):
        e = np.zeros(D)
        e[j] = 1.0
        out[:, j] = M.mult(e)
    return out


@pytest.mark.parametrize("two_s,n", [(1, 6), (2, 5), (3, 4), (4, 4)])
def test_measure_oracle_spin_s_operators_match_kronecker_products(two_s, n):
    """The oracle's digit-level site operators (measurements) equal the Kronecker-product operators of the
    spin-S Hamiltonian oracle on a random vector: <Sz_i>, <Sz_i Sz_j>, <S+_i S-_j>, <S-_i S+_j>."""
    from oracle import measure as omeasure
    from oracle import spin as ospin
    rng = np.random.default_rng(two_s * 10 + n)
    T = n * two_s // 2
    states = ospin.packed_states(n, two_s, T)
    psi = rng.normal(size=len(states))
    for ops in ([("Sz", 1)], [("Sz", 0), ("Sz", n - 1)], [("Sz", 2), ("Sz", 2)], [("Splus", 0), ("Sminus", 2)],
                [("Sminus", 1), ("Splus", 3)], [("Splus", 1), ("Sminus", 1)], [("Sminus", 2), ("Splus", 2)],
                [("Sz", 0), ("Splus", 1)]):
        got = omeasure._expect(states, psi, n, ops, two_s)
        ref = ospin.pair_expectation(n, two_s, T, psi, ops)
        assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)), (ops, got, ref)


def test_bloch_matrix_from_the_sector_matrix_equals_the_spin_half_restatement():
    """hamiltonian_from_sector (any site basis) on the spin-1/2 sector matrix gives the spin-1/2 Bloch
    matrix of bloch.hamiltonian at every momentum of an 8-site ring with nnn bonds and a field."""
    from oracle import spin as ospin
    n, n_up = 8, 4
    bonds = [(i, (i + 1) % n, 1.0, 0.8, 0.0) for i in range(n)] + [(i, (i + 2) % n, 0.3, 0.3, 0.0) for i in range(n)]
    h = [0.15] * n
    H = ospin.hamiltonian(n, 1, bonds, h, None, digit_sum=n_up)
    states = ospin.packed_states(n, 1, n_up)
    for k in bloch.translation_momenta("chain lattice", {"L": n}):
        tr = bloch.translations("chain lattice", {"L": n}, k)
        basis = bloch.bloch_basis(n, n_up, tr)
        M1 = bloch.hamiltonian(n, bonds, basis, site_h=h)
        M2 = bloch.hamiltonian_from_sector(H, states, basis)
        assert np.allclose(M1, M2, atol=1e-13)


@pytest.mark.parametrize("two_s,L", [(2, 6), (3, 4), (4, 4)])
def test_spin_s_momentum_sectors_partition_the_sz_spectrum(two_s, L):
    """Spin-S Bloch sectors (bloch_basis_of over packed digits): dimensions add up to the Sz sector's,
    and the union of the momentum spectra is its spectrum (ring with exchange, biquadratic, field and
    single-ion terms)."""
    from oracle import spin as ospin
    bits = two_s.bit_length()
    bonds = [(i, (i + 1) % L, 1.0, 0.9, 0.2) for i in range(L)]
    T = L * two_s // 2
    H = ospin.hamiltonian(L, two_s, bonds, [0.1] * L, [0.3] * L, digit_sum=T)
    states = ospin.packed_states(L, two_s, T)
    evs, dims = [], 0
    for k in bloch.translation_momenta("chain lattice", {"L": L}):
        tr = bloch.translations("chain lattice", {"L": L}, k)
        basis = bloch.bloch_basis_of(states, L, tr, lambda s, mp: bloch.translate_digits(s, mp, L, bits))
        dims += len(basis["reps"])
        if basis["reps"]:
            M = bloch.hamiltonian_from_sector(H, states, basis)
            evs += list(np.linalg.eigvals(M).real)
    assert dims == len(states)
    assert np.allclose(np.sort(evs), np.linalg.eigvalsh(H.toarray()), atol=1e-10)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_spin_s_oracle_at_spin_half_matches_example3_example4(seed):
    """The spin-S oracle's operator algebra (S+-, exchange_xy, biquadratic = (exchange_xy + Sz Sz)^2, site terms
    -h Sz + D Sz^2) at S = 1/2 reproduces the reference's HSpinBond (example3) and HSpinHalf (example4) at
    random couplings: rows/columns in the two-site product order (0,0), (0,1), (1,0), (1,1)."""
    from oracle import spin as ospin
    rng = np.random.default_rng(seed)
    jz, jxy, k, h, d = rng.uniform(-2, 2, 5)
    vals = {"Jz0": jz, "Jxy0": jxy, "K0": k, "h0": h, "D0": d, "Gamma0": 0.0}
    g4 = np.array(_nested_eval(gold("spin_half_example4.json")["HSpinHalf"], vals), dtype=float)
    H = ospin.hamiltonian(2, 1, [(0, 1, jz, jxy, k)], [h, h], [d, d]).toarray()
    np.testing.assert_allclose(H, g4, rtol=0, atol=1e-13)
    g3 = np.array(_nested_eval(gold("spin_terms_example3.json")["HSpinBond"], vals), dtype=float)
    B = ospin.hamiltonian(2, 1, [(0, 1, jz, jxy, k)]).toarray()
    for is1 in range(2):
        for is2 in range(2):
            for js1 in range(2):
                for js2 in range(2):
                    assert abs(B[(is1 << 1) | is2, (js1 << 1) | js2] - g3[is1][is2][js1][js2]) < 1e-13


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_spin_s_oracle_at_spin_one_matches_example4(seed):
    """The spin-S oracle at S = 1 (two sites, one bond with Jz, Jxy and biquadratic K, site terms h and D)
    equals the reference's HSpinOne (example4, local_S = 1) at random couplings; Gamma = 0 (the engine
    rejects it), so every remaining coefficient is printed exactly (0, 1, 2)."""
    from oracle import spin as ospin
    rng = np.random.default_rng(10 + seed)
    jz, jxy, k, h, d = rng.uniform(-2, 2, 5)
    vals = {"Jz0": jz, "Jxy0": jxy, "K0": k, "h0": h, "D0": d, "Gamma0": 0.0}
    g = np.array(_nested_eval(gold("spin_one_example4.json")["HSpinOne"], vals), dtype=float)
    H = ospin.hamiltonian(2, 2, [(0, 1, jz, jxy, k)], [h, h], [d, d]).toarray()
    np.testing.assert_allclose(H, g, rtol=0, atol=1e-12)
