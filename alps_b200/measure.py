"""Eigenvector measurements of an Sz sector: the MEASURE_* parameters of sparsediag.

Reference paths are relative to the ALPS source tree.

The parameters name the measurements (alps::MeasurementOperators,
src/alps/scheduler/measurement_operators.C:25-70):

  MEASURE_AVERAGE[name] = op            sum_i <op_i> / N
  MEASURE_LOCAL[name] = op              <op_i> for every site i
  MEASURE_CORRELATIONS[name] = "a:b"    <a_i b_j> (or "a" for a = b) per lattice distance
  MEASURE_STRUCTURE_FACTOR[name] = "a:b"  sum_ij <a_i b_j> cos(k.(r_j - r_i)) / N per momentum k

and DiagMatrix::perform_measurements (applications/diag/diag.h:191-314)
evaluates them in each eigenvector: a correlation takes, for every distance
class d, the first site pair (i outer, j inner) at that distance
(hypercubic_lattice::distance, src/alps/lattice/hypercubic.h:338-349: per
periodic direction (y - x) mod L, per open direction the pair itself), the
same site giving <a_i b_i>; the structure factor runs over the lattice's
momenta (hypercubic.h:371-387: cell order, k_d = 2 pi x_d / L_d with
x_d > L_d / 2 taken as x_d - L_d).  Operators: the spin-1/2 site operators
Sz, Splus, Sminus of the model's local spin (S = 1/2 .. 2, lib/xml/models.xml.in:24-36).
The expectation values come from aed_expectation (one pass over the vector
per 32 site pairs, on the GPU); this module only chooses the pairs and
combines the numbers.

In a momentum sector (translation invariance) perform_measurements skips the
local values, averages each correlation over all pairs of its distance class
(divided by the class's multiplicity, diag.h:236-258), and sums the
structure factor over all pairs; a class's pairs add up to a translation-
invariant operator, whose Bloch-basis expectation aed_momentum_expectation
returns, and e^{ik(r_j - r_i)} is the same for every pair of a class.
"""

from __future__ import annotations

import ctypes
import math
import re

import numpy as np

from . import AEDError, ERR_INVALID, _check, _dp, _I32P, _params_text, graph_of, lib

OBS_SZ, OBS_SZSZ, OBS_SPSM = 0, 1, 2
_SITE_OPS = ("Sz", "Splus", "Sminus")


def requests(params: dict) -> dict:
    """The MEASURE_* entries of a parameter dict: {"average": {name: op}, "local": {...},
    "correlations": {name: (a, b)}, "structure_factor": {name: (a, b)}}."""
    out = {"average": {}, "local": {}, "correlations": {}, "structure_factor": {}}
    for key, val in params.items():
        m = re.match(r"^MEASURE_(AVERAGE|LOCAL|CORRELATIONS|STRUCTURE_FACTOR)\[(.*)\]$", str(key))
        if not m:
            continue
        kind, name = m.group(1), m.group(2)
        v = str(val).strip().strip('"')
        if kind in ("AVERAGE", "LOCAL"):
            out["average" if kind == "AVERAGE" else "local"][name] = v
        else:
            pair = tuple(v.split(":", 1)) if ":" in v else (v, v)
            out["correlations" if kind == "CORRELATIONS" else "structure_factor"][name] = pair
    return out


class Geometry:
    """Sites, coordinates, distance classes and momenta of the lattice of a parameter set (a GRAPH: its
    vertices, their coordinates, one distance class per ordered pair, no momenta)."""

    def __init__(self, params):
        g = graph_of(params)
        self.graph = g is not None
        if self.graph:  # no lattice: every ordered site pair is its own distance class (graph_helper.h:516-582)
            self.n, self.dim, self.ext, self.periodic = g[0], 0, [], []
            self.coords = g.coords
            return
        dim, ext, per = ctypes.c_int32(0), (ctypes.c_int32 * 2)(), (ctypes.c_int32 * 2)()
        _check(lib().aed_lattice_geometry(_params_text(params).encode(), ctypes.byref(dim), ext, per))
        self.dim = dim.value
        self.ext = [ext[d] for d in range(self.dim)]
        self.periodic = [bool(per[d]) for d in range(self.dim)]
        self.n = int(np.prod(self.ext))
        self.coords = []
        for c in range(self.n):  # cell index: last coordinate fastest (hypercubic.h:181-209)
            cc, idx = [0] * self.dim, c
            for d in range(self.dim - 1, -1, -1):
                cc[d] = idx % self.ext[d]
                idx //= self.ext[d]
            self.coords.append(cc)

    def num_distances(self) -> int:
        if self.graph:
            return self.n * self.n
        d = 1
        for L, p in zip(self.ext, self.periodic):
            d *= L if p else L * L
        return d

    def distance(self, i: int, j: int) -> int:
        if self.graph:
            return i * self.n + j
        x, y = self.coords[i], self.coords[j]
        d = 0
        for a in range(self.dim):
            L = self.ext[a]
            if self.periodic[a]:
                d = d * L + (y[a] - x[a] if x[a] <= y[a] else L + y[a] - x[a])
            else:
                d = L * (d * L + x[a]) + y[a]
        return d

    def momenta(self):
        if self.graph:
            raise AEDError(ERR_INVALID, "structure factors need the momenta of a lattice: not on a GRAPH")
        out = []
        for cc in self.coords:
            k = []
            for a in range(self.dim):
                x, L = cc[a], self.ext[a]
                if x > L // 2:
                    x -= L
                k.append(2.0 * math.pi * x / L)
            out.append(k)
        return out


def _check_op(op):
    if op not in _SITE_OPS:
        raise AEDError(ERR_INVALID, f"measurement operator {op!r}: only the spin site operators "
                                    f"{', '.join(_SITE_OPS)} are supported")


def expectation(ham, psi, kind: int, si, sj=None) -> np.ndarray:
    """aed_expectation: <psi| O |psi> for the site pairs (si[p], sj[p])."""
    si = np.ascontiguousarray(si, dtype=np.int32)
    sj = np.ascontiguousarray(si if sj is None else sj, dtype=np.int32)
    out = np.zeros(max(si.size, 1))
    _check(lib().aed_expectation(ham._h, psi.ptr, kind, si.size, si.ctypes.data_as(_I32P), sj.ctypes.data_as(_I32P),
                                 _dp(out)))
    return out[:si.size]


def _site_values(ham, psi, op, n):
    _check_op(op)
    sites = np.arange(n)
    if op == "Sz":
        return expectation(ham, psi, OBS_SZ, sites)
    return np.zeros(n)  # S+ and S- change Sz: zero in an Sz sector


def _pair_values(ham, psi, a, b, si, sj):
    """<a_i b_j> for site pairs, the same site as the product a b of that site."""
    _check_op(a)
    _check_op(b)
    si, sj = np.asarray(si, dtype=np.int32), np.asarray(sj, dtype=np.int32)
    if a == "Sz" and b == "Sz":
        return expectation(ham, psi, OBS_SZSZ, si, sj)
    if (a, b) == ("Splus", "Sminus"):
        return expectation(ham, psi, OBS_SPSM, si, sj)
    if (a, b) == ("Sminus", "Splus"):
        # S-_i S+_j = S+_j S-_i for i != j; on one site S- S+ = S+ S- - 2 Sz
        v = expectation(ham, psi, OBS_SPSM, sj, si)
        same = si == sj
        if same.any():
            if getattr(ham, "two_s", 1) == 1:  # spin 1/2: S- S+ is the projector on spin down
                norm2 = expectation(ham, psi, OBS_SZSZ, si[same], si[same]) * 4.0  # |psi|^2
                v[same] = norm2 - v[same]
            else:
                v[same] = v[same] - 2.0 * expectation(ham, psi, OBS_SZ, si[same])
        return v
    return np.zeros(si.size)  # the product changes Sz: zero in an Sz sector


def momentum_sum(ham, psi, kind: int, si, sj=None) -> float:
    """aed_momentum_expectation: <psi| sum_p O(si[p], sj[p]) |psi> in a momentum sector."""
    si = np.ascontiguousarray(si, dtype=np.int32)
    sj = np.ascontiguousarray(si if sj is None else sj, dtype=np.int32)
    out = ctypes.c_double(0.0)
    _check(lib().aed_momentum_expectation(ham._h, psi.ptr, kind, si.size, si.ctypes.data_as(_I32P),
                                          sj.ctypes.data_as(_I32P), ctypes.byref(out)))
    return out.value


def _pair_sum(ham, psi, a, b, pairs) -> float:
    """Momentum sector: <sum over pairs of a_i b_j> (the same site as the product a b of that site)."""
    _check_op(a)
    _check_op(b)
    si = [p[0] for p in pairs]
    sj = [p[1] for p in pairs]
    if a == "Sz" and b == "Sz":
        return momentum_sum(ham, psi, OBS_SZSZ, si, sj)
    if (a, b) == ("Splus", "Sminus"):
        return momentum_sum(ham, psi, OBS_SPSM, si, sj)
    if (a, b) == ("Sminus", "Splus"):
        diff = [(i, j) for i, j in pairs if i != j]
        same = [i for i, j in pairs if i == j]
        v = momentum_sum(ham, psi, OBS_SPSM, [j for i, j in diff], [i for i, j in diff]) if diff else 0.0
        if same:
            if getattr(ham, "two_s", 1) == 1:  # S- S+ on one site: the projector on spin down, 1/2 - Sz
                v += 0.5 * len(same) - momentum_sum(ham, psi, OBS_SZ, same)
            else:  # S- S+ = S+ S- - 2 Sz on one site
                v += momentum_sum(ham, psi, OBS_SPSM, same, same) - 2.0 * momentum_sum(ham, psi, OBS_SZ, same)
        return v
    return 0.0


def _measure_momentum(ham, psi, req, g) -> dict:
    n = g.n
    out = {"average": {}, "local": {}, "correlations": {}, "structure_factor": {}}
    for name, op in req["average"].items():
        _check_op(op)
        out["average"][name] = momentum_sum(ham, psi, OBS_SZ, list(range(n))) / n if op == "Sz" else 0.0
    classes = {}
    for i in range(n):
        for j in range(n):
            classes.setdefault(g.distance(i, j), []).append((i, j))
    nd = g.num_distances()
    sums = {}
    for name, (a, b) in list(req["correlations"].items()) + list(req["structure_factor"].items()):
        if (a, b) not in sums:
            sums[(a, b)] = {d: _pair_sum(ham, psi, a, b, ps) for d, ps in classes.items()}
    for name, (a, b) in req["correlations"].items():
        row = [0.0] * nd
        for d, ps in classes.items():
            row[d] = sums[(a, b)][d] / len(ps)
        out["correlations"][name] = row
    if req["structure_factor"]:
        r = np.array(g.coords, dtype=float)
        ks = g.momenta()
        for name, (a, b) in req["structure_factor"].items():
            sk = []
            for k in ks:
                val = 0.0
                for d, ps in classes.items():
                    i, j = ps[0]
                    val += sums[(a, b)][d] * math.cos(float(np.dot(k, r[j] - r[i])))
                sk.append(val / n)
            out["structure_factor"][name] = sk
    return out


def measure(ham, psi, params, geometry: Geometry | None = None) -> dict:
    """The MEASURE_* quantities of params in the (normalised) device vector psi of a handle."""
    req = requests(params)
    if getattr(ham, "momentum", False):
        return _measure_momentum(ham, psi, req, geometry or Geometry(params))
    g = geometry or Geometry(params)
    n = g.n
    out = {"average": {}, "local": {}, "correlations": {}, "structure_factor": {}}
    for name, op in req["average"].items():
        out["average"][name] = float(np.sum(_site_values(ham, psi, op, n)) / n)
    for name, op in req["local"].items():
        out["local"][name] = _site_values(ham, psi, op, n).tolist()
    if req["correlations"]:
        first = {}
        for i in range(n):
            for j in range(n):
                first.setdefault(g.distance(i, j), (i, j))
        nd = g.num_distances()
        pairs = [first[d] for d in range(nd) if d in first]
        ds = [d for d in range(nd) if d in first]
        for name, (a, b) in req["correlations"].items():
            vals = _pair_values(ham, psi, a, b, [p[0] for p in pairs], [p[1] for p in pairs])
            row = [0.0] * nd
            for d, v in zip(ds, vals):
                row[d] = float(v)
            out["correlations"][name] = row
    if req["structure_factor"]:
        si = [i for i in range(n) for j in range(n)]
        sj = [j for i in range(n) for j in range(n)]
        ks = g.momenta()
        r = np.array(g.coords, dtype=float)
        for name, (a, b) in req["structure_factor"].items():
            c = _pair_values(ham, psi, a, b, si, sj).reshape(n, n)
            sk = []
            for k in ks:
                ph = r @ np.array(k)
                sk.append(float(np.sum(c * np.cos(ph[None, :] - ph[:, None])) / n))
            out["structure_factor"][name] = sk
    return out
