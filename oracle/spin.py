"""Oracle restatement of spin-S Sz sectors (S = 1/2 .. 2): basis order and the Hamiltonian.

TEST INFRASTRUCTURE ONLY: used by tests/ to check the engine's spin-S sectors
(alps_b200/csrc/spin.cu); the engine never imports this module.  scipy sparse
Kronecker products over the full Hilbert space, for small systems.

Restates (paths relative to the ALPS source tree):
  * the spin site basis: states Sz = -S .. S, S+ |m> = sqrt(S(S+1) - m(m+1)) |m+1>,
    S- |m> = sqrt(S(S+1) - m(m-1)) |m-1>          lib/xml/models.xml.in:24-36
  * the spin HAMILTONIAN: sum_i (-h_i Sz_i + D_i Sz_i^2) + sum_bonds (Jz Sz Sz
    + Jxy exchange_xy + K biquadratic), exchange_xy = (S+S- + S-S+)/2,
    biquadratic = (exchange_xy + Sz Sz)^2          models.xml.in:290-300, 342-373
  * basis order: site 0 most significant, last site fastest, the Sz_total
    constraint                                     src/alps/model/basisstates.h:175-278
The Kronecker product with site 0 as the first factor enumerates the full space
in exactly that order; the sector keeps the states of the requested Sz_total.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def site_ops(two_s: int):
    d = two_s + 1
    S = two_s / 2.0
    m = np.arange(d) - S
    sz = sp.diags(m)
    splus = sp.lil_matrix((d, d))
    for v in range(d - 1):
        splus[v + 1, v] = np.sqrt(S * (S + 1) - m[v] * (m[v] + 1))
    splus = splus.tocsr()
    return sz.tocsr(), splus, splus.T.tocsr()


def _embed(op, site, n, d):
    out = sp.identity(1, format="csr")
    for i in range(n):
        out = sp.kron(out, op if i == site else sp.identity(d, format="csr"), format="csr")
    return out


def sector(n: int, two_s: int, digit_sum: int) -> np.ndarray:
    """Indices (in the full space) of the sector's states in basis order, and their digit vectors."""
    d = two_s + 1
    idx = np.arange(d ** n)
    digits = np.array([(idx // d ** (n - 1 - i)) % d for i in range(n)]).T
    keep = digits.sum(axis=1) == digit_sum
    return idx[keep], digits[keep]


def hamiltonian(n: int, two_s: int, bonds, site_h=None, site_d=None, digit_sum=None):
    """Sparse H restricted to the sector of digit sum `digit_sum` (Sz_total + n S)."""
    d = two_s + 1
    sz, spl, smi = site_ops(two_s)
    dim = d ** n
    H = sp.csr_matrix((dim, dim))
    Z = [_embed(sz, i, n, d) for i in range(n)]
    P = [_embed(spl, i, n, d) for i in range(n)]
    M = [_embed(smi, i, n, d) for i in range(n)]
    for i in range(n):
        h = 0.0 if site_h is None else site_h[i]
        dd = 0.0 if site_d is None else site_d[i]
        if h or dd:
            H = H + (-h) * Z[i] + dd * (Z[i] @ Z[i])
    for b in bonds:
        i, j, jz, jxy = b[0], b[1], b[2], b[3]
        k = b[4] if len(b) > 4 else 0.0
        zz = Z[i] @ Z[j]
        xy = 0.5 * (P[i] @ M[j] + M[i] @ P[j])
        H = H + jz * zz + jxy * xy
        if k:
            x = xy + zz
            H = H + k * (x @ x)
    if digit_sum is None:
        return H.tocsr()
    keep, _ = sector(n, two_s, digit_sum)
    return H.tocsr()[keep][:, keep]


def packed_states(n: int, two_s: int, digit_sum: int) -> np.ndarray:
    """The sector's states packed as the engine stores them: ceil(log2(2S+1)) bits per site, site 0 first."""
    d = two_s + 1
    bits = 1
    while (1 << bits) < d:
        bits += 1
    _, digits = sector(n, two_s, digit_sum)
    out = np.zeros(len(digits), dtype=np.uint64)
    for i in range(n):
        out |= digits[:, i].astype(np.uint64) << np.uint64(bits * (n - 1 - i))
    return out


def pair_expectation(n: int, two_s: int, digit_sum: int, psi, ops) -> float:
    """<psi| ops[0] ops[1] ... |psi> in the sector of digit sum `digit_sum`, ops = [(name, site)] with
    name in Sz, Splus, Sminus (Kronecker-product operators over the full space, restricted)."""
    d = two_s + 1
    sz, spl, smi = site_ops(two_s)
    named = {"Sz": sz, "Splus": spl, "Sminus": smi}
    O = sp.identity(d ** n, format="csr")
    for name, site in ops:
        O = O @ _embed(named[name], site, n, d)
    keep, _ = sector(n, two_s, digit_sum)
    psi = np.asarray(psi, dtype=float)
    full = np.zeros(d ** n)
    full[keep] = psi
    return float(full @ (O @ full))
