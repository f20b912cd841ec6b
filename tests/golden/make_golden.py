"""Generate the golden fixtures in this folder from the reference's own test outputs.

Run in a checkout where the ALPS sources are available:

    python tests/golden/make_golden.py /path/to/alps

Reads (paths relative to the ALPS source tree) and writes JSON beside this script:
  test/model/example10.output   -> basis_example10.json  (2x2 square, all 16 states)
  test/model/example12.output   -> basis_example12.json  (2x2 square, Sz_total = 0)
  test/model/example3.output    -> spin_terms_example3.json (HSpinSite, HSpinBond)
  test/model/example4.output    -> spin_half_example4.json  (two-site HSpinHalf)
                                   spin_one_example4.json   (two-site HSpinOne, local_S = 1)
  test/lattice/label.output     -> labels_square4.json (4x4 square: site, bond, momentum, distance labels)
  test/lattice/example5.output  -> lattice_example5.json (anisotropic square 10x4 sites)
  test/lattice/example6.output  -> lattice_example6.json (anisotropic square 10x4 bonds)
  test/model/example13.output   -> bloch_example13.json (4-site chain, Bloch bases at k = 2 pi m / 4)
  test/model/example14.output   -> bloch_example14.json (2x2 square, k = (0, 0))
  test/model/example15.output   -> bloch_example15.json (2x2 square, every translation momentum)
The fixtures are committed; the tests never read the ALPS tree.
"""

from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _states(text):
    """Parse '[ |1/2 -1/2 > |1/2 1/2 > ... ]' rows into lists of Sz (as +1/-1)."""
    rows = []
    for line in text.splitlines():
        line = line.strip()
        if not line.startswith("["):
            continue
        kets = re.findall(r"\|\s*(\S+)\s+(\S+)\s*>", line)
        rows.append([1 if sz == "1/2" else -1 for _s, sz in kets])
    return rows


def _block(text, name):
    """Return the brace expression following 'name =' in an example output."""
    start = text.index(name)
    start = text.index("{", start)
    depth = 0
    for i in range(start, len(text)):
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                return text[start: i + 1]
    raise ValueError(name)


def _nested(expr):
    """'{{a, b}, {c, d}}' -> nested python lists of expression strings."""
    pos = 0

    def parse():
        nonlocal pos
        assert expr[pos] == "{"
        pos += 1
        items = []
        cur = ""
        while True:
            ch = expr[pos]
            if ch == "{":
                items.append(parse())
                cur = ""
            elif ch == ",":
                if cur.strip():
                    items.append(cur.strip())
                cur = ""
                pos += 1
            elif ch == "}":
                if cur.strip():
                    items.append(cur.strip())
                pos += 1
                return items
            else:
                cur += ch
                pos += 1

    return parse()


def _bloch_sections(text):
    """Split an example13-15 output into sections: translations (phase rounded to one digit, site
    map) and the built states (normalisation printed with 6 digits, Sz per site)."""
    sections = []
    cur = None
    for line in text.splitlines():
        m = re.match(r"Momentum:\s*(.*)$", line)
        if m:
            cur = {"momentum": [float(v) for v in m.group(1).split()], "translations": [], "states": []}
            sections.append(cur)
            continue
        m = re.match(r"Translation (\d+) with phase \(([-\d.e]+),([-\d.e]+)\) maps (.*)$", line)
        if m:
            if cur is None or (int(m.group(1)) == 0 and cur["states"]):
                cur = {"momentum": None, "translations": [], "states": []}
                sections.append(cur)
            mp = [int(b) for a, b in re.findall(r"(\d+)->(\d+)", m.group(4))]
            cur["translations"].append({"phase": [float(m.group(2)), float(m.group(3))], "map": mp})
            continue
        m = re.match(r"([-\d.e]+)\*\[(.*)\] \+ translations", line.strip())
        if m and cur is not None:
            kets = re.findall(r"\|\s*(\S+)\s+(\S+)\s*>", m.group(2))
            cur["states"].append({"norm": float(m.group(1)),
                                  "sz": [1 if sz == "1/2" else -1 for _s, sz in kets]})
    return sections


def main(alps):
    out = {}
    t = open(os.path.join(alps, "test/model/example10.output")).read()
    out["basis_example10.json"] = {
        "source": "test/model/example10.output",
        "lattice": "square lattice", "L": 2, "constraint": None,
        "states_sz": _states(t),
    }
    t = open(os.path.join(alps, "test/model/example12.output")).read()
    out["basis_example12.json"] = {
        "source": "test/model/example12.output",
        "lattice": "square lattice", "L": 2, "constraint": {"Sz_total": 0},
        "states_sz": _states(t),
    }
    t = open(os.path.join(alps, "test/model/example3.output")).read()
    out["spin_terms_example3.json"] = {
        "source": "test/model/example3.output",
        "HSpinSite": _nested(_block(t, "HSpinSite")),
        "HSpinBond": _nested(_block(t, "HSpinBond")),
    }
    t = open(os.path.join(alps, "test/model/example4.output")).read()
    out["spin_half_example4.json"] = {
        "source": "test/model/example4.output",
        "HSpinHalf": _nested(_block(t, "HSpinHalf")),
    }
    out["spin_one_example4.json"] = {
        "source": "test/model/example4.output",
        "HSpinOne": _nested(_block(t, "HSpinOne")),
    }
    t = open(os.path.join(alps, "test/lattice/label.output")).read()
    sec, lab = None, {}
    for line in t.splitlines():
        if line.endswith("labels:"):
            sec = line[:-len(" labels:")].lower()
            lab[sec] = []
        elif sec and line.strip():
            lab[sec].append(line.strip())
    out["labels_square4.json"] = {
        "source": "test/lattice/label.output",
        "params": {"LATTICE": "square lattice", "L": 4},
        "sites": lab["site"], "bonds": lab["bond"], "momenta": lab["momenta"], "distances": lab["distance"],
    }
    t = open(os.path.join(alps, "test/lattice/example5.output")).read()
    sites = []
    for m in re.finditer(r"Site (\d+) has type (\d+) and has coordinates ([\d\s\.\-]+)", t):
        sites.append({"site": int(m.group(1)), "type": int(m.group(2)),
                      "coords": [float(v) for v in m.group(3).split()]})
    out["lattice_example5.json"] = {
        "source": "test/lattice/example5.output",
        "params": {"LATTICE": "anisotropic square lattice", "L": 10, "W": 4},
        "sites": sites,
    }
    t = open(os.path.join(alps, "test/lattice/example6.output")).read()
    bonds = [[int(a), int(b), int(c)] for a, b, c in
             re.findall(r"The bond between site (\d+) and site (\d+) has type (\d+)", t)]
    out["lattice_example6.json"] = {
        "source": "test/lattice/example6.output",
        "params": {"LATTICE": "anisotropic square lattice", "L": 10, "W": 4},
        "bonds": bonds,
    }
    for ex, lat, L in (("13", "chain lattice", 4), ("14", "square lattice", 2), ("15", "square lattice", 2)):
        t = open(os.path.join(alps, f"test/model/example{ex}.output")).read()
        out[f"bloch_example{ex}.json"] = {
            "source": f"test/model/example{ex}.output",
            "lattice": lat, "L": L, "constraint": None,
            "sections": _bloch_sections(t),
        }
    for name, obj in out.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(obj, f, indent=1)
        print("wrote", name)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <ALPS source tree>")
    main(sys.argv[1])
