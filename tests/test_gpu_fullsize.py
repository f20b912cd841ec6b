"""Parity at the full benchmark sizes (needs a B200).

The J1-J2 chain L=28 (D = 40,116,600; J2 from the seed-2802 stream) and the 6x5
square lattice with per-bond J ~ U[0.8, 1.2] (seed 3005; D = 155,117,520) are
too large for the oracle's whole explicit matrix, so the oracle builds the
explicit rows of sampled windows only (``oracle.rows_mult``, the reference's
element order and lower_bound lookups over the full sector): the first rows,
the middle of the sector, the last rows, and seeded random windows.  FP64 rows
of every apply variant must equal them bit for bit; FP32 rows must lie within
2 eps32 * sum_j |M_ij x_j| of the exact row of the rounded input.
"""

from math import comb

import numpy as np
import pytest

import alps_b200 as ed
import oracle

pytestmark = pytest.mark.gpu

EPS32 = np.finfo(np.float32).eps
WINDOW = 16384


def chain_bonds(L, j2):
    out = []
    for i in range(L):
        out.append((i, (i + 1) % L, 1.0, 1.0, 0.0))
        out.append((i, (i + 2) % L, float(j2), float(j2), 0.0))
    return out


def square_bonds(Lx, Wy, seed):
    raw = []
    for x in range(Lx):
        for y in range(Wy):
            s = x * Wy + y
            raw.append((s, x * Wy + (y + 1) % Wy))
            raw.append((s, ((x + 1) % Lx) * Wy + y))
    js = np.random.default_rng(seed).uniform(0.8, 1.2, len(raw))
    return [(a, b, float(j), float(j), 0.0) for (a, b), j in zip(raw, js)]


CASES = {
    "l28_j1j2": (28, 14, lambda: chain_bonds(28, np.random.default_rng(2802).uniform(0.0, 0.5))),
    "sq6x5": (30, 15, lambda: square_bonds(6, 5, 3005)),
}


def windows(D, seed):
    rng = np.random.default_rng(seed)
    starts = [0, D // 2 - WINDOW // 2, D - WINDOW] + sorted(int(v) for v in rng.integers(0, D - WINDOW, 3))
    return [(s, s + WINDOW) for s in starts]


@pytest.fixture(scope="module", params=sorted(CASES))
def sector(request):
    N, n_up, mk = CASES[request.param]
    bonds = mk()
    states = oracle.basis_fast(N, n_up)
    assert states.size == comb(N, n_up)
    x = np.random.default_rng(N).normal(size=states.size)
    wins = windows(states.size, N + 1)
    ref = {w: oracle.rows_mult(N, states, bonds, x, *w) for w in wins}
    x32 = x.astype(np.float32).astype(np.float64)
    ref32 = {w: oracle.rows_mult(N, states, bonds, x32, *w) for w in wins}
    return {"name": request.param, "N": N, "n_up": n_up, "bonds": bonds, "states": states, "x": x,
            "x32": x32, "wins": wins, "ref": ref, "ref32": ref32}


def _variants(ham, xd, yd):
    out = []
    for v in range(len(ed.apply_variants())):
        try:
            ham.time_apply(xd, yd, 1, v)
            out.append(v)
        except ed.AEDError:
            pass
    return out


def test_fullsize_fp64_rows_bit_exact_every_variant(sector):
    """FP64 H x at full size: every apply variant's rows in the sampled windows equal the explicit
    matrix's rows bit for bit (hamiltonian_matrix.hpp:307-345, ublas.h:57-63)."""
    ham = ed.Hamiltonian(sector["N"], sector["n_up"], sector["bonds"], precision=ed.FP64)
    assert ham.dim == sector["states"].size
    xd, yd = ham.new_vector().upload(sector["x"]), ham.new_vector()
    vs = _variants(ham, xd, yd)
    assert vs, "no apply variant fits"
    for v in vs:
        ham.time_apply(xd, yd, 1, v)
        y = yd.download()
        for w in sector["wins"]:
            got = y[w[0]:w[1]]
            exp = sector["ref"][w][0]
            bad = np.flatnonzero(got != exp)
            assert bad.size == 0, (ed.apply_variants()[v], w, bad[:5] + w[0], got[bad[:5]], exp[bad[:5]])
    xd.free()
    yd.free()
    ham.close()


def test_fullsize_fp32_rows_within_bound_every_variant(sector):
    """FP32 H x at full size: rows within 2 eps32 sum_j |M_ij x_j| of the exact rows of the rounded x,
    and every variant gives the same rows."""
    ham = ed.Hamiltonian(sector["N"], sector["n_up"], sector["bonds"], precision=ed.FP32)
    xd, yd = ham.new_vector().upload(sector["x32"]), ham.new_vector()
    vs = _variants(ham, xd, yd)
    assert vs
    first = None
    for v in vs:
        ham.time_apply(xd, yd, 1, v)
        y = yd.download()
        cut = np.concatenate([y[w[0]:w[1]] for w in sector["wins"]])
        if first is None:
            first = cut
            for w in sector["wins"]:
                exp, absrow = sector["ref32"][w]
                err = np.abs(y[w[0]:w[1]] - exp)
                assert np.all(err <= 2 * EPS32 * absrow + 1e-30), (w, float(np.max(err / (absrow + 1e-300))))
        else:
            assert np.array_equal(cut, first), ed.apply_variants()[v]
    xd.free()
    yd.free()
    ham.close()


@pytest.mark.parametrize("N,k", [(28, 14), (30, 15)])
def test_fullsize_basis_windows_equal_oracle(N, k):
    """basis_states order at N = 28, 30: windows of the engine's basis equal the oracle's enumeration,
    and their ranks are the window's indices (basisstates.h:68-74, 175-278)."""
    ham = ed.Hamiltonian(N, k, [(0, 1, 1.0, 1.0)])
    ref = oracle.basis_fast(N, k)
    D = ref.size
    assert ham.dim == D
    rng = np.random.default_rng(N)
    offs = [0, D // 2, D - 4096] + [int(v) for v in rng.integers(0, D - 4096, 5)]
    for o in offs:
        got = ham.basis(o, 4096)
        assert np.array_equal(got, ref[o:o + 4096]), o
        assert np.array_equal(ham.index(got), np.arange(o, o + 4096))
    ham.close()
