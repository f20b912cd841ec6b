"""Parity of the CUDA engine against the oracle, through the C ABI (needs a B200)."""

from math import comb

import numpy as np
import pytest

import alps_b200 as ed
import oracle
from oracle import lattice

pytestmark = pytest.mark.gpu

EPS32 = np.finfo(np.float32).eps


def spin_params(**kw):
    p = {"MODEL": "spin", "CONSERVED_QUANTUMNUMBERS": "Sz", "TRANSLATION_SYMMETRY": "false", "Sz_total": 0}
    p.update(kw)
    return p


def random_bonds(lat, params, seed, lo=0.5, hi=1.5):
    """ALPS bonds of a lattice with per-bond couplings drawn uniformly."""
    n, _, bonds = lattice.lattice_graph(lat, params)
    rng = np.random.default_rng(seed)
    js = rng.uniform(lo, hi, len(bonds))
    return n, [(s, t, float(j), float(j), 0.0) for (s, t, _), j in zip(bonds, js)]


# ---------------------------------------------------------------- basis / rank
@pytest.mark.parametrize("N,k", [(2, 1), (4, 2), (5, 0), (5, 5), (9, 4), (16, 8), (17, 9), (20, 10), (24, 12)])
def test_basis_bit_exact(N, k):
    ham = ed.Hamiltonian(N, k, [(0, 1, 1.0, 1.0)])
    assert ham.dim == comb(N, k)
    ref = oracle.basis(N, k)
    got = ham.basis()
    assert np.array_equal(got, ref)
    idx = ham.index(ref)
    assert np.array_equal(idx, np.arange(ham.dim))


def test_index_outside_sector_returns_dimension():
    ham = ed.Hamiltonian(10, 5, [(0, 1, 1.0, 1.0)])
    bad = np.array([0, 1, 0b1111100001, (1 << 10) | 0b11111, 0xffffffff], dtype=np.uint32)
    assert np.all(ham.index(bad) == ham.dim)


@pytest.mark.parametrize("N,k", [(28, 14), (30, 15), (32, 16)])
def test_basis_full_size_properties(N, k):
    """Size-independent checks at the largest sectors: sorted, popcount, count, rank round trip."""
    ham = ed.Hamiltonian(N, k, [(0, 1, 1.0, 1.0)])
    D = ham.dim
    assert D == comb(N, k)
    rng = np.random.default_rng(N)
    offs = np.unique(np.concatenate([[0, D - 4096], rng.integers(0, D - 4096, 16)]))
    for o in offs:
        st = ham.basis(int(o), 4096)
        assert np.all(np.diff(st.astype(np.int64)) > 0)
        pc = np.unpackbits(st.view(np.uint8)).reshape(-1, 32).sum(1)
        assert np.all(pc == k)
        assert np.array_equal(ham.index(st), np.arange(o, o + 4096))
    if N < 32:
        assert ham.basis(0, 1)[0] == (1 << k) - 1
        assert ham.basis(D - 1, 1)[0] == ((1 << k) - 1) << (N - k)


# ---------------------------------------------------------------- H x, FP64
HV_CASES = [
    ("chain16", dict(LATTICE="chain lattice", L=16, J=1)),
    ("nnn18", dict(LATTICE="nnn chain lattice", L=18, J=1, J1=0.4137)),
    ("square4x4", dict(LATTICE="square lattice", L=4, J=1)),
    ("ladder8", dict(LATTICE="ladder", L=8, J0=0.93, J1=1.27)),
    ("open_chain_h", dict(LATTICE="open chain lattice", L=14, J=1, h=0.3, D=0.2)),
    ("xxz", dict(LATTICE="chain lattice", L=14, Jz=1.7, Jxy=0.45)),
    ("nnn4_dup", dict(LATTICE="nnn chain lattice", L=4, J=1, J1=0.7)),
    ("chain2_dup", dict(LATTICE="chain lattice", L=2, J=1)),
    ("sz1", dict(LATTICE="chain lattice", L=15, J=1, Sz_total=0.5)),
    ("biquad", dict(LATTICE="chain lattice", L=12, J=1, K0=0.3)),
]


def _oracle_for(m):
    return oracle.Matrix(m["n_sites"], m["n_up"], m["bonds"], site_h=m["site_h"], site_d=m["site_d"])


@pytest.mark.parametrize("name,p", HV_CASES, ids=[c[0] for c in HV_CASES])
def test_hv_fp64_bit_exact_against_explicit_matrix(name, p):
    ham = ed.Hamiltonian.from_parameters(spin_params(**p))
    M = _oracle_for(ham.params)
    assert M.D == ham.dim
    rng = np.random.default_rng(1)
    for _ in range(2):
        x = rng.normal(size=ham.dim)
        y = ham.apply(x)
        ref = M.mult(x)
        assert np.array_equal(y, ref), np.max(np.abs(y - ref))


@pytest.mark.parametrize("seed", [0, 1])
def test_hv_fp64_bit_exact_random_bond_square_4x5(seed):
    n, bonds = random_bonds("square lattice", {"L": 4, "W": 5}, seed, 0.8, 1.2)
    ham = ed.Hamiltonian(n, n // 2, bonds)
    M = oracle.Matrix(n, n // 2, bonds)
    x = np.random.default_rng(seed).normal(size=ham.dim)
    assert np.array_equal(ham.apply(x), M.mult(x))


def _apply_variants(ham):
    """Indices of the apply variants that fit this sector (tile and bundle kernels)."""
    x, y = ham.new_vector(), ham.new_vector()
    ham.fill_random(x, 1)
    out = []
    for v in range(len(ed.apply_variants())):
        try:
            ham.time_apply(x, y, 1, v)
            out.append(v)
        except ed.AEDError:
            pass
    return out


VARIANT_CASES = [HV_CASES[0], HV_CASES[1], HV_CASES[4], HV_CASES[6], HV_CASES[7], HV_CASES[8], HV_CASES[9],
                 ("square4x4_h", dict(LATTICE="square lattice", L=4, J=1, h=0.21))]


@pytest.mark.parametrize("name,p", VARIANT_CASES, ids=[c[0] for c in VARIANT_CASES])
def test_hv_every_variant_fp64_bit_exact(name, p):
    """Every apply variant (tile and bundle kernels, forced) gives the explicit matrix's rows bit for bit."""
    ham = ed.Hamiltonian.from_parameters(spin_params(**p))
    M = _oracle_for(ham.params)
    x = np.random.default_rng(11).normal(size=ham.dim)
    ref = M.mult(x)
    xd, yd = ham.new_vector().upload(x), ham.new_vector()
    vs = _apply_variants(ham)
    assert len(vs) >= 12
    for v in vs:
        yd.upload(np.full(ham.dim, np.nan))
        ham.time_apply(xd, yd, 1, v)
        assert np.array_equal(yd.download(), ref), (v, ed.lib().aed_last_error())


@pytest.mark.parametrize("seed", [0, 1])
def test_hv_every_variant_random_square_4x5(seed):
    n, bonds = random_bonds("square lattice", {"L": 4, "W": 5}, seed, 0.8, 1.2)
    for prec in (ed.FP64, ed.FP32):
        ham = ed.Hamiltonian(n, n // 2, bonds, precision=prec)
        x = np.random.default_rng(seed).normal(size=ham.dim)
        xd, yd = ham.new_vector().upload(x), ham.new_vector()
        outs = []
        for v in _apply_variants(ham):
            ham.time_apply(xd, yd, 1, v)
            outs.append(yd.download())
        for o in outs[1:]:
            assert np.array_equal(o, outs[0])
        if prec == ed.FP64:
            assert np.array_equal(outs[0], oracle.Matrix(n, n // 2, bonds).mult(x))


@pytest.mark.parametrize("prec", [ed.FP64, ed.FP32])
def test_lanczos_step_alpha_identical_across_variants(prec, monkeypatch):
    """The fused <x, y> partials and |w| are formed in a fixed order: alpha and beta agree bit for
    bit whichever apply variant the autotuner picks."""
    n, bonds = random_bonds("square lattice", {"L": 4, "W": 5}, 7, 0.8, 1.2)
    rng = np.random.default_rng(8)
    got = []
    probe = ed.Hamiltonian(n, n // 2, bonds, precision=prec)
    vs = _apply_variants(probe)
    v0 = rng.normal(size=probe.dim)
    v0 /= np.linalg.norm(v0)
    probe.close()
    for v in vs:
        monkeypatch.setenv("AED_HV_VARIANT", str(v))
        ham = ed.Hamiltonian(n, n // 2, bonds, precision=prec)
        cur, nxt = ham.new_vector().upload(v0), ham.new_vector()
        got.append((ham.lanczos_step(None, cur, nxt, 0.0), nxt.download()))
        ham.close()
    for (ab, w) in got[1:]:
        assert ab == got[0][0]
        assert np.array_equal(w, got[0][1])


def _fp32_bound(M, x):
    rp, col, val = M.csr()
    absrow = np.add.reduceat(np.abs(val) * np.abs(x[col]), rp[:-1])
    return absrow


@pytest.mark.parametrize("name,p", HV_CASES[:5], ids=[c[0] for c in HV_CASES[:5]])
def test_hv_fp32_compensated_within_bound(name, p):
    """FP32 vectors: y_i within 2 eps32 * sum_j |M_ij x_j| of the exact FP64 row (tolerance of the test)."""
    ham = ed.Hamiltonian.from_parameters(spin_params(**p), precision=ed.FP32)
    M = _oracle_for(ham.params)
    x = np.random.default_rng(3).normal(size=ham.dim).astype(np.float32).astype(np.float64)
    y = ham.apply(x)
    ref = M.mult(x)
    bound = 2 * EPS32 * _fp32_bound(M, x) + 1e-30
    assert np.all(np.abs(y - ref) <= bound)


def test_hv_full_size_sum_rule_square_6x5():
    """6x5 square lattice (D = 155,117,520), per-bond J: 1^T H 1 in closed form (FP64)
    and the symmetry <u, H z> = <H u, z> (FP32 handle)."""
    n, bonds = random_bonds("square lattice", {"L": 6, "W": 5}, 3005, 0.8, 1.2)
    D_anti = 2 * comb(n - 2, 14)
    ham64 = ed.Hamiltonian(n, 15, bonds, precision=ed.FP64)
    D = ham64.dim
    assert D == 155117520
    # every bond: D_anti antiparallel rows (-Jz/4 on the diagonal, Jxy/2 off it),
    # D - D_anti parallel rows (+Jz/4)
    expect = sum(b[2] / 4 * (D - 2 * D_anti) + b[3] / 2 * D_anti for b in bonds)
    one = ham64.new_vector().upload(np.ones(D))
    h1 = ham64.new_vector()
    ham64.mult(one, h1)
    assert ham64.dot(one, h1) == pytest.approx(expect, rel=1e-12)
    one.free()
    h1.free()
    ham64.close()
    ham = ed.Hamiltonian(n, 15, bonds, precision=ed.FP32)
    u, z, hu, hz = (ham.new_vector() for _ in range(4))
    ham.fill_random(u, 11)
    ham.fill_random(z, 7)
    ham.mult(u, hu)
    ham.mult(z, hz)
    lhs, rhs = ham.dot(u, hz), ham.dot(hu, z)
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


# ---------------------------------------------------------------- vector ops
@pytest.mark.parametrize("prec", [ed.FP64, ed.FP32])
def test_vector_ops_against_numpy(prec):
    ham = ed.Hamiltonian.from_parameters(spin_params(LATTICE="chain lattice", L=14, J=1), precision=prec)
    D = ham.dim
    rng = np.random.default_rng(0)
    xh, yh = rng.normal(size=D), rng.normal(size=D)
    if prec == ed.FP32:
        xh, yh = xh.astype(np.float32).astype(float), yh.astype(np.float32).astype(float)
    x, y = ham.new_vector().upload(xh), ham.new_vector().upload(yh)
    assert ham.dot(x, y) == pytest.approx(float(xh @ yh), rel=1e-12)
    assert ham.two_norm(x) == pytest.approx(float(np.linalg.norm(xh)), rel=1e-12)
    ham.axpy(0.5, x, y)
    tol = 1e-15 if prec == ed.FP64 else 1e-6
    np.testing.assert_allclose(y.download(), yh + 0.5 * xh, rtol=tol, atol=tol)
    ham.scal(3.0, x)
    np.testing.assert_allclose(x.download(), 3 * xh, rtol=tol)
    ham.div(3.0, x)
    np.testing.assert_allclose(x.download(), xh, rtol=tol)
    z = ham.new_vector()
    ham.copy(x, z)
    assert np.array_equal(z.download(), x.download())
    ham.fill_random(z, 42)
    st = oracle.start_vector(42, D)
    if prec == ed.FP64:
        assert np.array_equal(z.download(), st)
    else:
        assert np.all(np.abs(z.download() - st) < 2 ** -23)
    assert ham.dot(z, z) == ham.dot(z, z)


def test_lanczos_step_matches_numpy():
    ham = ed.Hamiltonian.from_parameters(spin_params(LATTICE="nnn chain lattice", L=14, J=1, J1=0.3))
    M = _oracle_for(ham.params)
    D = ham.dim
    rng = np.random.default_rng(4)
    v0 = rng.normal(size=D)
    v0 /= np.linalg.norm(v0)
    v1 = rng.normal(size=D)
    v1 -= (v1 @ v0) * v0
    v1 /= np.linalg.norm(v1)
    a_prev = ham.new_vector().upload(v0)
    cur = ham.new_vector().upload(v1)
    nxt = ham.new_vector()
    beta_prev = 0.37
    a, b = ham.lanczos_step(a_prev, cur, nxt, beta_prev)
    w = M.mult(v1)
    a_ref = v1 @ w
    w = w - a_ref * v1 - beta_prev * v0
    b_ref = np.linalg.norm(w)
    assert a == pytest.approx(a_ref, rel=1e-13)
    assert b == pytest.approx(b_ref, rel=1e-13)
    np.testing.assert_allclose(nxt.download(), w / b_ref, atol=1e-13)


# ---------------------------------------------------------------- solves
SOLVE_CASES = [
    ("cfg1_chain16", dict(LATTICE="chain lattice", L=16, J=1), 4),
    ("nnn16", dict(LATTICE="nnn chain lattice", L=16, J=1, J1=0.241), 2),
    ("ladder7", dict(LATTICE="ladder", L=7, J0=1.13, J1=0.61), 3),
    ("square4x4", dict(LATTICE="square lattice", L=4, J=1), 2),
    ("sz1_chain15", dict(LATTICE="chain lattice", L=15, J=1, Sz_total=0.5), 2),
]


@pytest.mark.parametrize("name,p,nev", SOLVE_CASES, ids=[c[0] for c in SOLVE_CASES])
def test_solve_fp64_matches_oracle(name, p, nev):
    ham = ed.Hamiltonian.from_parameters(spin_params(**p))
    M = _oracle_for(ham.params)
    r = ham.solve(nev=nev, seed=9)
    o = M.lanczos(nev=nev, seed=9)
    assert r["converged"]
    assert len(r["evals"]) == len(o["evals"])
    np.testing.assert_allclose(r["evals"], o["evals"], rtol=1e-12, atol=1e-12)
    assert np.all(r["errors"] <= np.maximum(100 * np.finfo(float).eps,
                                            100 * np.finfo(float).eps * np.abs(r["evals"])))
    if ham.dim <= 4000:
        w = np.linalg.eigvalsh(M.dense())
        np.testing.assert_allclose(r["evals"][0], w[0], rtol=1e-12)


def test_solve_matches_oracle_alpha_beta_start():
    """Same start vector: the first alpha/beta agree with the oracle's recurrence to rounding.  The
    partial sums of <x, y> and |w| are grouped differently from the oracle's sequential sums, so the two
    recurrences part at the rounding level and the stop can come a few iterations apart (the bound:
    a tenth of the count plus 3); the eigenvalues agree."""
    ham = ed.Hamiltonian.from_parameters(spin_params(LATTICE="chain lattice", L=16, J=1))
    M = _oracle_for(ham.params)
    r = ham.solve(nev=2, seed=123)
    o = M.lanczos(nev=2, seed=123)
    a, b = ham.last_tmatrix()
    n = 10
    np.testing.assert_allclose(a[:n], o["alpha"][:n], rtol=1e-11)
    np.testing.assert_allclose(b[:n], o["beta"][:n], rtol=1e-10)
    assert abs(r["iterations"] - o["iterations"]) <= 0.1 * o["iterations"] + 3
    np.testing.assert_allclose(r["evals"][:2], o["evals"][:2], rtol=1e-12)


def test_solve_deterministic():
    ham = ed.Hamiltonian.from_parameters(spin_params(LATTICE="nnn chain lattice", L=18, J=1, J1=0.2))
    r1 = ham.solve(nev=2, seed=5)
    a1, b1 = ham.last_tmatrix()
    r2 = ham.solve(nev=2, seed=5)
    a2, b2 = ham.last_tmatrix()
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)
    assert np.array_equal(r1["evals"], r2["evals"])


def test_solve_closed_forms():
    # dimer and 4-site ring
    r = ed.Hamiltonian(2, 1, [(0, 1, 1.0, 1.0)]).solve(nev=1)
    assert abs(r["evals"][0] + 0.75) < 1e-14
    ham = ed.Hamiltonian.from_parameters(spin_params(LATTICE="chain lattice", L=4, J=1))
    assert abs(ham.solve(nev=1)["evals"][0] + 2.0) < 1e-13


def test_solve_dimension_one_and_max_iter():
    ham = ed.Hamiltonian.from_parameters(spin_params(LATTICE="chain lattice", L=6, J=1, Sz_total=3))
    assert ham.dim == 1
    r = ham.solve(nev=2)
    assert r["evals"].tolist() == [1.5]
    ham = ed.Hamiltonian.from_parameters(spin_params(LATTICE="chain lattice", L=16, J=1))
    r = ham.solve(nev=4, max_iter=5)
    assert not r["converged"] and r["iterations"] == 5


def test_majumdar_ghosh_full_size_L28():
    """Config-2 lattice (nnn chain L=28, D=40,116,600) at J2 = J1/2: E0 = -3 L / 8 exactly."""
    ham = ed.Hamiltonian.from_parameters(spin_params(LATTICE="nnn chain lattice", L=28, J=1, J1=0.5))
    assert ham.dim == 40116600
    r = ham.solve(nev=1, seed=1)
    assert r["converged"]
    assert abs(r["evals"][0] + 10.5) < 1e-12 * 10.5


# ---------------------------------------------------------------- mixed precision
MIXED_CASES = [
    ("chain16", dict(LATTICE="chain lattice", L=16, J=1), 4),
    ("nnn20", dict(LATTICE="nnn chain lattice", L=20, J=1, J1=0.33), 2),
    ("ladder9", dict(LATTICE="ladder", L=9, J0=1.21, J1=0.77), 2),
]


@pytest.mark.parametrize("name,p,nev", MIXED_CASES, ids=[c[0] for c in MIXED_CASES])
def test_mixed_precision_within_1e9_of_fp64(name, p, nev):
    p = spin_params(**p)
    h64 = ed.Hamiltonian.from_parameters(p)
    h32 = ed.Hamiltonian.from_parameters(p, precision=ed.FP32)
    r64 = h64.solve(nev=nev, seed=2)
    r32 = h32.solve(nev=nev, seed=2)
    assert r64["converged"] and r32["converged"]
    assert len(r32["evals"]) == len(r64["evals"])
    rel = np.abs(r32["evals"] - r64["evals"]) / np.abs(r64["evals"])
    assert np.all(rel <= 1e-9), rel
    assert r32["iterations_low"] > 0


@pytest.mark.parametrize("name,p,nev", MIXED_CASES, ids=[c[0] for c in MIXED_CASES])
def test_mixed_refinements_agree(name, p, nev):
    """Both FP64 refinements of the FP32 phase -- Rayleigh-Ritz over its Ritz vectors (the default)
    and FP64 Lanczos from their combination (refine=1) -- land within 1e-9 of the FP64 solve, and the
    Rayleigh-Ritz error bound it reports holds against the FP64 values."""
    p = spin_params(**p)
    r64 = ed.Hamiltonian.from_parameters(p).solve(nev=nev, seed=2)
    h32 = ed.Hamiltonian.from_parameters(p, precision=ed.FP32)
    rr = h32.solve(nev=nev, seed=2)
    lz = h32.solve(nev=nev, seed=2, refine=1)
    # the default takes Rayleigh-Ritz when its bound holds and FP64 Lanczos otherwise
    assert rr["refined_by"] in ("rayleigh_ritz", "lanczos"), rr
    assert lz["refined_by"] == "lanczos"
    for r in (rr, lz):
        assert r["converged"] and len(r["evals"]) == len(r64["evals"])
        assert np.all(np.abs(r["evals"] - r64["evals"]) <= 1e-9 * np.abs(r64["evals"]))
    if rr["refined_by"] == "rayleigh_ritz":
        # the Rayleigh-Ritz values lie above the true ones by at most the bound (plus FP64 rounding)
        d = rr["evals"] - r64["evals"]
        assert np.all(d >= -1e-12 * np.abs(r64["evals"]))
        assert np.all(d <= rr["errors"] + 1e-12 * np.abs(r64["evals"]))


@pytest.mark.parametrize("L,j2", [(20, 0.2), (22, 0.3)])
def test_rayleigh_ritz_refinement_taken_on_a_gapped_ground_state(L, j2):
    """A J1-J2 chain's ground state (a clear gap to the next level): the FP32 phase's Ritz vector refined
    by Rayleigh-Ritz alone (K FP64 applies, no FP64 Lanczos steps), within 1e-9 of the FP64 solve."""
    p = spin_params(LATTICE="nnn chain lattice", L=L, J=1, J1=j2)
    r64 = ed.Hamiltonian.from_parameters(p).solve(nev=1, seed=4)
    r32 = ed.Hamiltonian.from_parameters(p, precision=ed.FP32).solve(nev=1, seed=4)
    assert r32["refined_by"] == "rayleigh_ritz", r32
    assert r32["iterations"] <= 6  # the FP64 applies of the refinement
    assert abs(r32["evals"][0] - r64["evals"][0]) <= 1e-9 * abs(r64["evals"][0])


@pytest.mark.parametrize("nev", [3, 4])
def test_rayleigh_ritz_with_ghost_copies_in_the_clusters(nev):
    """Heisenberg chain L=22 (uniform J): the FP32 phase runs long enough for a ghost copy of the ground
    state, so the Ritz vectors of the nev lowest clusters (K > nev) hold a nearly dependent pair.  The
    Rayleigh-Ritz step still bounds the nev lowest pairs (the pair made of the copy's FP32 noise lies
    above the gap and is left out), and every value agrees with the FP64 solve within its reported
    bound and 1e-9."""
    b = [(i, (i + 1) % 22, 1.0, 1.0, 0.0) for i in range(22)]
    r64 = ed.Hamiltonian(22, 11, b).solve(nev=nev, seed=2)
    r32 = ed.Hamiltonian(22, 11, b, precision=ed.FP32).solve(nev=nev, seed=2)
    assert r32["refined_by"] == "rayleigh_ritz", r32
    assert r32["iterations"] > nev  # K Ritz vectors: the clusters held a ghost copy
    assert len(r32["evals"]) == nev == len(r64["evals"])
    for e32, e64, err in zip(r32["evals"], r64["evals"], r32["errors"]):
        assert abs(e32 - e64) <= 1e-9 * abs(e64)
        assert e32 - e64 <= err + 1e-12 * abs(e64)  # the bound holds (values from above)


def test_reserved_basis_store_gives_the_same_solve():
    """aed_reserve_basis sizes the FP32 basis store ahead (here for more vectors than the solve takes,
    and for fewer): the mixed solve's values, errors and iteration counts equal those of a handle whose
    store grew inside the solve, bit for bit; the FP64 handle, which keeps no basis, refuses."""
    b = [(i, (i + 1) % 20, 1.0, 1.0, 0.0) for i in range(20)] + [(i, (i + 2) % 20, 0.3, 0.3, 0.0) for i in range(20)]
    grown = ed.Hamiltonian(20, 10, b, precision=ed.FP32)
    r0 = grown.solve(nev=2, seed=5)
    for n in (300, 20):
        h = ed.Hamiltonian(20, 10, b, precision=ed.FP32)
        h.reserve_basis(n)
        r = h.solve(nev=2, seed=5)
        for k in ("evals", "errors"):
            assert np.array_equal(r[k], r0[k]), (n, k)
        assert (r["iterations"], r["iterations_low"]) == (r0["iterations"], r0["iterations_low"])
        h.close()
    grown.close()
    h64 = ed.Hamiltonian(20, 10, b)
    with pytest.raises(ed.AEDError, match="basis"):
        h64.reserve_basis(16)
    h64.close()


def _basis_and_copies(ham, r):
    """The stored FP32 Lanczos basis V (m x D) of the last mixed solve, max |V V^T - I|, and how many
    eigenvalues of its T-matrix lie within 1e-5 relative of the lowest (1 + the ghost copies)."""
    m = r["iterations_low"] + 1
    V = np.array([ham.lanczos_vector(j) for j in range(m)])
    orth = float(np.max(np.abs(V @ V.T - np.eye(m))))
    a, b = ham.last_tmatrix(fp32_phase=True)
    T = np.diag(a) + np.diag(b[:-1], 1) + np.diag(b[:-1], -1)
    w = np.linalg.eigvalsh(T)
    return orth, int(np.sum(np.abs(w - w[0]) <= 1e-5 * abs(w[0])))


def test_full_reorthogonalisation_of_the_fp32_basis():
    """Option reorth (FP32 handles): every FP32 Lanczos vector is reorthogonalised against the stored basis.
    The basis stays orthonormal to FP32 rounding (|V V^T - I| <= 1e-5) where plain Lanczos loses it, the
    T-matrix holds one copy of the ground state (plain Lanczos run as long makes ghost copies), and the
    eigenvalues still agree with the FP64 solve to 1e-9."""
    p = spin_params(LATTICE="square lattice", L=4, J=1)
    r64 = ed.Hamiltonian.from_parameters(p).solve(nev=6, seed=3)
    h32 = ed.Hamiltonian.from_parameters(p, precision=ed.FP32)
    plain = h32.solve(nev=6, seed=3)
    orth0, copies0 = _basis_and_copies(h32, plain)
    ro = h32.solve(nev=6, seed=3, reorth=True)
    orth1, copies1 = _basis_and_copies(h32, ro)
    assert orth1 <= 1e-5, orth1
    assert copies1 == 1, copies1
    assert orth0 > 10 * orth1 and copies0 >= copies1, (orth0, copies0)
    for r in (plain, ro):
        assert r["converged"] and len(r["evals"]) == len(r64["evals"])
        assert np.all(np.abs(r["evals"] - r64["evals"]) <= 1e-9 * np.abs(r64["evals"]))
    with pytest.raises(ed.AEDError):
        ed.Hamiltonian.from_parameters(p).solve(nev=1, reorth=True)  # FP64 handles store no basis


@pytest.mark.parametrize("L,seed", [(22, 2), (24, 2), (24, 5)])
def test_mixed_precision_near_degenerate_pair(L, seed):
    """J1-J2 chain near the Majumdar-Ghosh point (J2 = 0.49972474): the two lowest states are
    split by ~1e-6 relative, below what the FP32 phase resolves.  The FP64 refinement must still
    return both, as the plain FP64 path does (1e-9 relative, both eigenvalues)."""
    n = L
    bonds = []
    for i in range(n):
        bonds.append((i, (i + 1) % n, 1.0, 1.0))
        bonds.append((i, (i + 2) % n, 0.49972474, 0.49972474))
    h64 = ed.Hamiltonian(n, n // 2, bonds)
    h32 = ed.Hamiltonian(n, n // 2, bonds, precision=ed.FP32)
    r64 = h64.solve(nev=2, seed=seed)
    r32 = h32.solve(nev=2, seed=seed)
    assert r64["converged"] and r32["converged"]
    assert r64["evals"][1] - r64["evals"][0] < 1e-4  # the pair is resolved by FP64
    rel = np.abs(r32["evals"] - r64["evals"]) / np.abs(r64["evals"])
    assert np.all(rel <= 1e-9), (r32["evals"], r64["evals"])


def test_set_couplings_matches_fresh_handle():
    """aed_set_couplings re-targets a handle: same results as a handle built from scratch."""
    p1 = spin_params(LATTICE="nnn chain lattice", L=14, J=1, J1=0.2)
    p2 = spin_params(LATTICE="nnn chain lattice", L=14, J=1, J1=0.45, h=0.1)
    ham = ed.Hamiltonian.from_parameters(p1)
    m2 = ed.model_from_parameters(p2)
    ham.set_couplings(m2["bonds"], m2["site_h"], m2["site_d"])
    ref = _oracle_for(m2)
    x = np.random.default_rng(2).normal(size=ham.dim)
    assert np.array_equal(ham.apply(x), ref.mult(x))
    with pytest.raises(ed.AEDError):
        ham.set_couplings([(0, 1, 1.0, 1.0)] * 3 + [(0, 15, 1.0, 1.0)])


@pytest.mark.parametrize("prec", [ed.FP64, ed.FP32])
def test_handles_reuse_cached_memory(prec):
    """Handles created after others were destroyed take their memory from the per-process cache: every
    solve of the loop gives the same eigenvalues and recurrence length, before and after empty_cache."""
    n, bonds = random_bonds("square lattice", {"L": 4, "W": 5}, 3, 0.8, 1.2)
    got = []
    for k in range(4):
        if k == 2:
            ed.empty_cache(0)
        ham = ed.Hamiltonian(n, n // 2, bonds, precision=prec)
        r = ham.solve(nev=2, seed=5)
        ham.close()
        got.append((list(r["evals"]), r["iterations"]))
    assert all(g == got[0] for g in got[1:])
    with pytest.raises(ed.AEDError):
        ed.empty_cache(99)
