"""Oracle restatement of ALPS momentum (Bloch) sectors for spin models.

TEST INFRASTRUCTURE ONLY: used by tests/ to check the engine's momentum
sectors; the engine has its own implementation (alps_b200/csrc/momentum.cu,
model.cpp) and never imports this module.  Pure Python: for the small sectors
the tests use (up to ~16 sites).

Restates (paths relative to the ALPS source tree):
  * translation momenta, periodic directions in order, the first slowest
                                        src/alps/lattice/hypercubic.h:395-423
  * translations with their phases exp(i k.R), the first periodic direction
    fastest; one vertex per cell     hypercubic.h:425-464, latticegraph.h:252-269
  * the Bloch basis: states in basis order, an orbit's first state is its
    representative, kept when sqrt|sum of the phases of the translations that
    fix it| >= 0.01, normalisation that value / sqrt(number of sites); every
    other state maps to its representative through the first translation that
    reaches it                         src/alps/model/blochbasisstates.h:92-271
  * matrix elements: M(i, j) += val * phase * n_j / n_i for the image of
    representative i under a site or bond term, site terms before bonds
                                       src/alps/model/hamiltonian_matrix.hpp:268-291,
                                       307-345, 385-397
  * the TOTAL_MOMENTUM label: write_vector with 20 significant digits
                                       src/alps/utility/vectorio.hpp:170-180
States are integers with site i at bit n-1-i and spin up = 1, so that integer
order is the reference's basis order (site 0 most significant, index 0 = down);
spin-S states pack the digit m + S of every site in `bits` bits the same way
(bloch_basis_of, translate_digits, hamiltonian_from_sector).
Pinned by tests/golden/bloch_example13/14/15.json (the reference's
test/model/example13-15.output).
"""

from __future__ import annotations

import cmath
import math

import numpy as np

from .lattice import _LATTICES, _extents


def _geometry(name: str, params: dict):
    cell, ext_spec, bnd = _LATTICES[name]
    ext = _extents(ext_spec, params)
    return ext, bnd


def periodic_dirs(name: str, params: dict):
    ext, bnd = _geometry(name, params)
    return [d for d in range(len(ext)) if bnd[d] == "periodic"]


def translation_momenta(name: str, params: dict):
    """hypercubic_lattice::translation_momenta: list of k vectors (one entry per periodic direction)."""
    ext, bnd = _geometry(name, params)
    ks = []
    for i in range(len(ext)):
        if bnd[i] != "periodic":
            continue
        if not ks:
            ks = [[2.0 * j * math.pi / ext[i]] for j in range(ext[i])]
        else:
            ks = [k + [2.0 * j * math.pi / ext[i]] for k in ks for j in range(ext[i])]
    return [tuple(k) for k in ks]


def momentum_label(k) -> str:
    """alps::write_vector(k) with the default delimiter and 20 significant digits."""
    return " ".join("%.20g" % v for v in k)


def translations(name: str, params: dict, k):
    """hypercubic_lattice::translations(k): [(phase, site map)], translation t moving site i to map[i]."""
    ext, bnd = _geometry(name, params)
    dim = len(ext)
    dirs = [d for d in range(dim) if bnd[d] == "periodic"]
    if len(k) != len(dirs):
        raise ValueError("one momentum component per periodic direction")
    n = 1
    for e in ext:
        n *= e

    def coords(idx):
        c = [0] * dim
        for d in range(dim - 1, -1, -1):
            c[d] = idx % ext[d]
            idx //= ext[d]
        return c

    def index(c):
        idx = 0
        for d in range(dim):
            idx = idx * ext[d] + c[d]
        return idx

    shift = [0] * len(dirs)
    out = []
    while True:
        off = [0] * dim
        phase = 0.0
        for i, d in enumerate(dirs):
            off[d] = shift[i]
            phase += shift[i] * float(k[i])
        mp = []
        for c in range(n):
            cc = coords(c)
            mp.append(index([(cc[d] + off[d]) % ext[d] for d in range(dim)]))
        out.append((cmath.exp(complex(0.0, phase)), mp))
        done = True
        for i in range(len(shift)):
            shift[i] += 1
            if shift[i] >= ext[dirs[i]]:
                shift[i] = 0
            else:
                done = False
                break
        if done:
            break
    return out


def translate(state: int, mp, n: int) -> int:
    out = 0
    for i in range(n):
        if (state >> (n - 1 - i)) & 1:
            out |= 1 << (n - 1 - mp[i])
    return out


def translate_digits(state: int, mp, n: int, bits: int) -> int:
    """A translation of a spin-S state packed with `bits` bits per site (site 0 most significant)."""
    out = 0
    mask = (1 << bits) - 1
    for i in range(n):
        out |= ((state >> (bits * (n - 1 - i))) & mask) << (bits * (n - 1 - mp[i]))
    return out


def bloch_basis(n: int, n_up, trans):
    """bloch_basis_states::build for spin-1/2 sites (n_up = None: no Sz constraint).

    Returns dict(reps=[state], norm=[float], rep_of={state: (representative index, phase)})."""
    states = (s for s in range(1 << n) if n_up is None or bin(s).count("1") == n_up)
    return bloch_basis_of(states, n, trans, lambda s, mp: translate(s, mp, n))


def bloch_basis_of(states, n: int, trans, translate_fn):
    """bloch_basis_states::build over `states` in basis order (any site basis whose states translate
    with translate_fn(state, site map))."""
    l = math.sqrt(float(n))
    reps, norm = [], []
    rep_of = {}
    for s in states:
        s = int(s)
        rep_number = None
        ph = 1.0 + 0.0j
        phase_sum = 1.0 + 0.0j
        for phase, mp in trans[1:]:
            t = translate_fn(s, mp)
            if t > s:
                continue
            if t == s:
                phase_sum += phase
                continue
            hit = rep_of.get(t)
            if hit is not None and reps[hit[0]] == t:
                rep_number = hit[0]
                ph = phase
                break
        store = True
        if rep_number is None:
            w = math.sqrt(abs(phase_sum))
            if w < 0.01:
                store = False
            else:
                rep_number = len(reps)
                norm.append(w / l)
                reps.append(s)
        if store:
            rep_of[s] = (rep_number, ph)
    return {"reps": reps, "norm": norm, "rep_of": rep_of}


def hamiltonian(n: int, bonds, basis, site_h=None, site_d=None) -> np.ndarray:
    """Dense complex M of the Bloch basis (site terms, then bonds in order)."""
    reps, norm, rep_of = basis["reps"], basis["norm"], basis["rep_of"]
    dim = len(reps)
    M = np.zeros((dim, dim), dtype=complex)

    def add(i, new_state, val):
        hit = rep_of.get(new_state)
        if hit is None:
            return
        j, phase = hit
        M[i, j] += val * (phase * norm[j] / norm[i])

    for i, r in enumerate(reps):
        if site_h is not None or site_d is not None:
            for s in range(n):
                h = 0.0 if site_h is None else site_h[s]
                d = 0.0 if site_d is None else site_d[s]
                up = (r >> (n - 1 - s)) & 1
                val = 0.25 * d - 0.5 * h if up else 0.25 * d + 0.5 * h
                if val != 0.0:
                    add(i, r, val)
        for b in bonds:
            s1, s2, jz, jxy = b[0], b[1], b[2], b[3]
            kq = b[4] if len(b) > 4 else 0.0
            m1, m2 = 1 << (n - 1 - s1), 1 << (n - 1 - s2)
            a, c = (r & m1) != 0, (r & m2) != 0
            if a == c:
                if 0.25 * jz + 0.0625 * kq != 0.0:
                    add(i, r, 0.25 * jz + 0.0625 * kq)
                continue
            # target site states in the order (0,0), (0,1), (1,0), (1,1) of the loop over js1, js2
            terms = [(r, -0.25 * jz + 0.3125 * kq), (r ^ m1 ^ m2, 0.5 * jxy - 0.25 * kq)]
            for new_state, val in (terms[::-1] if a else terms):
                if val != 0.0:
                    add(i, new_state, val)
    return M


def hamiltonian_from_sector(H, states, basis) -> np.ndarray:
    """Dense complex M of the Bloch basis from the sector's real matrix H over `states` (basis order):
    M(i, j) += <s|H|r_i> * phase * n_j / n_i for every state s with H[s, r_i] != 0 that maps to
    representative j (hamiltonian_matrix.hpp:307-345; any site basis)."""
    reps, norm, rep_of = basis["reps"], basis["norm"], basis["rep_of"]
    index = {int(s): k for k, s in enumerate(states)}
    Hc = H.tocsc()
    M = np.zeros((len(reps), len(reps)), dtype=complex)
    for i, r in enumerate(reps):
        col = index[int(r)]
        for k in range(Hc.indptr[col], Hc.indptr[col + 1]):
            hit = rep_of.get(int(states[Hc.indices[k]]))
            if hit is None:
                continue
            j, phase = hit
            M[i, j] += Hc.data[k] * (phase * norm[j] / norm[i])
    return M
