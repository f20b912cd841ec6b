"""Oracle restatement of sparsediag's eigenvector measurements for spin-S Sz sectors.

TEST INFRASTRUCTURE ONLY: used by tests/ to check alps_b200.measure; the
engine never imports this module.  Pure Python / numpy on explicit basis
lists, for small sectors.

Restates (paths relative to the ALPS source tree):
  * MEASURE_* parameter parsing          src/alps/scheduler/measurement_operators.C:25-70
  * perform_measurements: averages sum_i <op_i>/N, local <op_i>, correlations
    at the first site pair of each distance class, structure factor
    sum_ij Re(<a_i b_j> conj(e^{i k r_i}) e^{i k r_j}) / N
                                         applications/diag/diag.h:191-314
  * distance classes                     src/alps/lattice/hypercubic.h:325-349
  * momenta (cell order, x > L/2 -> x - L)  hypercubic.h:371-387
  * spin site operators: Sz |m> = m |m>, S+ |m> = sqrt(S(S+1) - m(m+1)) |m+1>,
    S- |m> = sqrt(S(S+1) - m(m-1)) |m-1>  lib/xml/models.xml.in:24-36 (spin 1/2: S+ |down> = |up>)
States are integers with site i at bit n-1-i, up = 1 (the basis order); for
spin S the digit m + S of site i at bits (n-1-i) b .., b bits per site.
"""

from __future__ import annotations

import math
import re

import numpy as np

from .lattice import _LATTICES, _extents


def requests(params: dict) -> dict:
    out = {"average": {}, "local": {}, "correlations": {}, "structure_factor": {}}
    for key, val in params.items():
        m = re.match(r"^MEASURE_(AVERAGE|LOCAL|CORRELATIONS|STRUCTURE_FACTOR)\[(.*)\]$", str(key))
        if not m:
            continue
        v = str(val).strip().strip('"')
        if m.group(1) == "AVERAGE":
            out["average"][m.group(2)] = v
        elif m.group(1) == "LOCAL":
            out["local"][m.group(2)] = v
        else:
            pair = tuple(v.split(":", 1)) if ":" in v else (v, v)
            out["correlations" if m.group(1) == "CORRELATIONS" else "structure_factor"][m.group(2)] = pair
    return out


def _geometry(params):
    _, ext_spec, bnd = _LATTICES[params["LATTICE"]]
    ext = _extents(ext_spec, params)
    n = int(np.prod(ext))
    coords = []
    for c in range(n):
        cc = []
        for d in range(len(ext) - 1, -1, -1):
            cc.append(c % ext[d])
            c //= ext[d]
        coords.append(cc[::-1])
    return ext, [b == "periodic" for b in bnd], coords


def _distance(ext, per, x, y):
    d = 0
    for a, L in enumerate(ext):
        if per[a]:
            d = d * L + ((y[a] - x[a]) % L)
        else:
            d = L * (d * L + x[a]) + y[a]
    return d


def _num_distances(ext, per):
    return int(np.prod([L if p else L * L for L, p in zip(ext, per)]))


def _op_apply(op, site, n, s, two_s=1):
    """op acting on site of state s: (coefficient, new state) or None.  Spin S = two_s / 2: the
    site's digit v = m + S sits at bits (n-1-site) * b .. with b = bits per site (1 for spin 1/2,
    where v is the up bit); S+ |m> = sqrt(S(S+1) - m(m+1)) |m+1>, S- |m> = sqrt(S(S+1) - m(m-1)) |m-1>."""
    b = two_s.bit_length()  # enough bits for the digits 0 .. 2S
    w = b * (n - 1 - site)
    v = (s >> w) & ((1 << b) - 1)
    S = two_s / 2.0
    m = v - S
    if op == "Sz":
        return m, s
    if op == "Splus":
        return (math.sqrt(S * (S + 1) - m * (m + 1)), s + (1 << w)) if v < two_s else None
    if op == "Sminus":
        return (math.sqrt(S * (S + 1) - m * (m - 1)), s - (1 << w)) if v > 0 else None
    raise ValueError(op)


def _expect(states, psi, n, ops, two_s=1):
    """<psi| ops[0] ops[1] ... |psi> with ops = [(name, site)], the rightmost acting first."""
    index = {int(s): k for k, s in enumerate(states)}
    tot = 0.0
    for k, s in enumerate(states):
        s, c = int(s), 1.0
        for name, site in reversed(ops):
            r = _op_apply(name, site, n, s, two_s)
            if r is None:
                c = 0.0
                break
            c *= r[0]
            s = r[1]
        if c != 0.0 and s in index:
            tot += c * psi[index[s]] * psi[k]
    return tot


def measure(states, psi, params, two_s=1) -> dict:
    """The MEASURE_* quantities in the vector psi over the basis `states` (spin S = two_s / 2: states
    packed as aed_spin_basis lists them)."""
    ext, per, coords = _geometry(params)
    n_sites = len(coords)
    req = requests(params)

    def ex(ops):
        return _expect(states, psi, n_sites, ops, two_s)

    out = {"average": {}, "local": {}, "correlations": {}, "structure_factor": {}}
    for name, op in req["average"].items():
        out["average"][name] = sum(ex([(op, i)]) for i in range(n_sites)) / n_sites
    for name, op in req["local"].items():
        out["local"][name] = [ex([(op, i)]) for i in range(n_sites)]
    nd = _num_distances(ext, per)
    for name, (a, b) in req["correlations"].items():
        row, done = [0.0] * nd, [False] * nd
        for i in range(n_sites):
            for j in range(n_sites):
                d = _distance(ext, per, coords[i], coords[j])
                if not done[d]:
                    row[d] = ex([(a, i), (b, j)])
                    done[d] = True
        out["correlations"][name] = row
    for name, (a, b) in req["structure_factor"].items():
        c = np.array([[ex([(a, i), (b, j)]) for j in range(n_sites)]
                      for i in range(n_sites)])
        ks = []
        for cc in coords:
            k = []
            for a_, L in enumerate(ext):
                x = cc[a_]
                if x > L // 2:
                    x -= L
                k.append(2.0 * math.pi * x / L)
            ks.append(k)
        sk = []
        for k in ks:
            val = 0.0
            for i in range(n_sites):
                for j in range(n_sites):
                    p1 = sum(k[d] * coords[i][d] for d in range(len(ext)))
                    p2 = sum(k[d] * coords[j][d] for d in range(len(ext)))
                    val += (c[i, j] * np.conj(complex(math.cos(p1), math.sin(p1))) *
                            complex(math.cos(p2), math.sin(p2))).real / n_sites
            sk.append(val)
        out["structure_factor"][name] = sk
    return out


def measure_translation_invariant(states, psi, params, two_s=1) -> dict:
    """perform_measurements with translation invariance (diag.h:213, 236-258): no local values, each
    correlation the mean over all site pairs of its distance class; averages and structure factors as
    in measure()."""
    ext, per, coords = _geometry(params)
    n_sites = len(coords)
    out = measure(states, psi, {k: v for k, v in params.items() if not str(k).startswith("MEASURE_CORRELATIONS")
                                and not str(k).startswith("MEASURE_LOCAL")}, two_s)
    req = requests(params)
    nd = _num_distances(ext, per)
    for name, (a, b) in req["correlations"].items():
        tot, cnt = [0.0] * nd, [0] * nd
        for i in range(n_sites):
            for j in range(n_sites):
                d = _distance(ext, per, coords[i], coords[j])
                tot[d] += _expect(states, psi, n_sites, [(a, i), (b, j)], two_s)
                cnt[d] += 1
        out["correlations"][name] = [t / c if c else 0.0 for t, c in zip(tot, cnt)]
    return out
