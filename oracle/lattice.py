"""Oracle restatement of the ALPS lattice library and spin-model parameter defaults.

TEST INFRASTRUCTURE ONLY: used by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of bench.py to check the engine; the engine has its own C++
implementation (alps_b200/csrc/model.cpp) and never imports this module.

Restates (paths relative to the ALPS source tree):
  * lattice graphs and unit cells      lib/xml/lattices.xml.in:170-211, 326-346,
                                       416-450, 470-516
  * cell index (last coordinate fastest) src/alps/lattice/hypercubic.h:181-209
  * edge generation, cell by cell in unit-cell edge order, self-loops dropped
                                       src/alps/lattice/latticegraph.h:98-136
  * spin HAMILTONIAN parameter defaults lib/xml/models.xml.in:342-373
Pinned by tests/golden/lattice_example5.json / lattice_example6.json (the
reference's test/lattice/example5.output and example6.output).
"""

from __future__ import annotations

# unit cells: list of (source offset, target offset, edge type)
_UNITCELLS = {
    "simple1d": [((0,), (1,), 0)],
    "complex1d": [((0,), (1,), 0), ((0,), (2,), 1)],
    "simple2d": [((0, 0), (0, 1), 0), ((0, 0), (1, 0), 0)],
    "anisotropic2d": [((0, 0), (1, 0), 0), ((0, 0), (0, 1), 1)],
}

# name -> (unit cell, extents as parameter names with defaults, boundaries)
_LATTICES = {
    "chain lattice": ("simple1d", ("L",), ("periodic",)),
    "open chain lattice": ("simple1d", ("L",), ("open",)),
    "nnn chain lattice": ("complex1d", ("L",), ("periodic",)),
    "nnn open chain lattice": ("complex1d", ("L",), ("open",)),
    "square lattice": ("simple2d", ("L", "W=L"), ("periodic", "periodic")),
    "open square lattice": ("simple2d", ("L", "W=L"), ("open", "open")),
    "anisotropic square lattice": ("anisotropic2d", ("L", "W=L"), ("periodic", "periodic")),
    "ladder": ("anisotropic2d", ("L", "W=2"), ("periodic", "open")),
    "open ladder": ("anisotropic2d", ("L", "W=2"), ("open", "open")),
}


def _extents(spec, params):
    out = []
    for item in spec:
        if "=" in item:
            name, default = item.split("=")
            val = params.get(name)
            if val is None:
                val = params[default] if default in params else int(default)
        else:
            val = params[item]
        out.append(int(val))
    return out


def lattice_graph(name: str, params: dict):
    """Return (n_sites, coords, bonds) with bonds as [(source, target, type)] in ALPS order."""
    cell, ext_spec, bnd = _LATTICES[name]
    ext = _extents(ext_spec, params)
    edges = _UNITCELLS[cell]
    dim = len(ext)
    n_cells = 1
    for e in ext:
        n_cells *= e

    def cell_coords(idx):
        c = [0] * dim
        for d in range(dim - 1, -1, -1):  # last coordinate fastest
            c[d] = idx % ext[d]
            idx //= ext[d]
        return c

    def cell_index(c):
        idx = 0
        for d in range(dim):
            idx = idx * ext[d] + c[d]
        return idx

    def shift(c, off):
        out = []
        for d in range(dim):
            v = c[d] + off[d]
            if v < 0 or v >= ext[d]:
                if bnd[d] == "open":
                    return None
                v %= ext[d]
            out.append(v)
        return out

    coords = [cell_coords(i) for i in range(n_cells)]
    bonds = []
    for ci in range(n_cells):
        c = coords[ci]
        for src_off, tgt_off, etype in edges:
            s = shift(c, src_off)
            t = shift(c, tgt_off)
            if s is None or t is None:
                continue
            si, ti = cell_index(s), cell_index(t)
            if si != ti:
                bonds.append((si, ti, etype))
    return n_cells, coords, bonds


def _num(v):
    if isinstance(v, (int, float)):
        return float(v)
    v = str(v).strip().strip('"')
    if "/" in v:
        a, b = v.split("/")
        return float(a) / float(b)
    return float(v)


def resolve_coupling(params: dict, bond_type: int):
    """(Jz, Jxy, K) for a bond type, following the HAMILTONIAN "spin" defaults.

    HAMILTONIAN parameters (models.xml.in:343-358): J0=0, J=J0, Jz=J, Jxy=J,
    Jz0=Jz, Jxy0=Jxy, J1=0, J'=J1, Jz'=J', Jxy'=J', Jz1=Jz', Jxy1=Jxy'.
    BONDTERM parameters (models.xml.in:366-371): J#=0, Jz#=J#, Jxy#=J#, K#=0,
    with '#' the bond type.
    """
    p = {k: v for k, v in params.items()}

    def get(name, chain):
        if name in p:
            return _num(p[name])
        for nxt in chain:
            if nxt in p:
                return _num(p[nxt])
        return None

    defaults = {
        "J0": "0", "J": "J0", "Jz": "J", "Jxy": "J", "Jz0": "Jz", "Jxy0": "Jxy",
        "J1": "0", "J'": "J1", "Jz'": "J'", "Jxy'": "J'", "Jz1": "Jz'", "Jxy1": "Jxy'",
        "K": "0",
    }

    def value(name):
        seen = set()
        while True:
            if name in p:
                return _num(p[name])
            if name in seen:
                return 0.0
            seen.add(name)
            d = defaults.get(name)
            if d is None:
                return None
            try:
                return float(d)
            except ValueError:
                name = d

    t = str(bond_type)
    jz = value("Jz" + t)
    if jz is None:  # Jz# = J#, J# = 0
        jz = value("J" + t)
        if jz is None:
            jz = 0.0
    jxy = value("Jxy" + t)
    if jxy is None:
        jxy = value("J" + t)
        if jxy is None:
            jxy = 0.0
    k = value("K" + t)
    if k is None:
        k = 0.0
    return jz, jxy, k


def spin_model(params: dict):
    """Map an ALPS parameter dict to (N, n_up, bonds[(s1, s2, Jz, Jxy, K)])."""
    n, _, bonds = lattice_graph(params["LATTICE"], params)
    out = []
    for s1, s2, t in bonds:
        jz, jxy, k = resolve_coupling(params, t)
        out.append((s1, s2, jz, jxy, k))
    szt = _num(params.get("Sz_total", 0))
    n_up = int(round(n / 2 + szt))
    return n, n_up, out
