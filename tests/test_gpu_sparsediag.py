"""The sparsediag task: the loop over Sz sectors (DiagMatrix::dostep), the ground state and
gap over sectors and the XML output, against dense spectra of the oracle (needs a B200)."""

import xml.etree.ElementTree as ET

import numpy as np
import pytest

import oracle
from alps_b200 import sparsediag

pytestmark = pytest.mark.gpu

PARAMS = {"MODEL": "spin", "LATTICE": "nnn chain lattice", "L": 8, "J": 1, "J1": 0.3,
          "CONSERVED_QUANTUMNUMBERS": "Sz", "TRANSLATION_SYMMETRY": "false", "NUMBER_EIGENVALUES": 2}


def dense_levels(n_up):
    from oracle import lattice
    N, _, bonds = lattice.spin_model(dict(PARAMS, Sz_total=n_up - 4))
    w = np.linalg.eigvalsh(oracle.Matrix(N, n_up, bonds).dense())
    distinct = [w[0]]
    for v in w[1:]:
        if v - distinct[-1] > 1e-9:
            distinct.append(v)
    return np.array(distinct)


def test_all_sz_sectors_ground_state_and_gap(tmp_path):
    res = sparsediag.run(PARAMS)
    secs = res["sectors"]
    assert [s["quantumnumbers"][0][1] for s in secs] == [str(k) for k in range(-4, 5)]
    for k, s in enumerate(secs):
        ref = dense_levels(k)
        n = min(2, ref.size)
        assert s["energies"].size == n
        np.testing.assert_allclose(s["energies"], ref[:n], rtol=1e-12, atol=1e-12)
    all_levels = np.sort(np.concatenate([dense_levels(k)[:2] for k in range(9)]))
    assert res["ground_state_energy"] == pytest.approx(all_levels[0], rel=1e-12)
    # the reference's gap: the next value over the sectors' lowest two (sparsediag.h:62-76)
    assert res["energy_gap"] == pytest.approx(all_levels[1] - all_levels[0], rel=1e-9, abs=1e-12)
    out = tmp_path / "spectrum.xml"
    sparsediag.write_xml(res, str(out), PARAMS)
    root = ET.parse(out).getroot()
    ev = root.findall("EIGENVALUES")
    assert len(ev) == 9
    assert ev[4].find("QUANTUMNUMBER").get("name") == "Sz" and ev[4].find("QUANTUMNUMBER").get("value") == "0"
    text = (ev[4].text or "") + "".join(c.tail or "" for c in ev[4])  # the values follow QUANTUMNUMBER
    np.testing.assert_allclose([float(v) for v in text.split()], secs[4]["energies"], rtol=0, atol=0)
    names = [a.get("name") for a in root.find("AVERAGES")]
    assert names == ["Ground State Energy", "Energy Gap"]


def test_fixed_sector_and_half_integer_labels():
    res = sparsediag.run(dict(PARAMS, Sz_total=0))
    assert len(res["sectors"]) == 1 and res["sectors"][0]["quantumnumbers"] == []
    odd = sparsediag.run(dict(PARAMS, LATTICE="chain lattice", L=5, NUMBER_EIGENVALUES=1))
    assert [s["quantumnumbers"][0][1] for s in odd["sectors"]] == ["-5/2", "-3/2", "-1/2", "1/2", "3/2", "5/2"]


def test_sparsediag_on_a_graph_of_a_lattice_library(tmp_path):
    """A <GRAPH> of a lattice library (10 vertices of two types, edges of three types in file order): every Sz
    sector's ground state equals the oracle's dense spectrum of the same bonds and site terms (1e-10)."""
    n = 10
    edges = [(i, (i + 1) % n, 0) for i in range(n)] + [(i, (i + 3) % n, 1) for i in range(0, n, 2)] + \
        [(0, 5, 2), (2, 7, 2)]
    vt = [i % 2 for i in range(n)]
    xml = ['<LATTICES>', f'<GRAPH name="test graph" vertices="{n}">']
    xml += [f'  <VERTEX id="{i + 1}" type="{t}"/>' for i, t in enumerate(vt)]
    xml += [f'  <EDGE type="{t}" source="{s + 1}" target="{d + 1}"/>' for s, d, t in edges]
    xml += ['</GRAPH>', '</LATTICES>']
    f = tmp_path / "g.xml"
    f.write_text("\n".join(xml))
    J = {0: (1.0, 0.9), 1: (0.4, 0.4), 2: (0.7, 1.1)}
    h = {0: 0.05, 1: -0.1}
    p = {"MODEL": "spin", "LATTICE_LIBRARY": str(f), "LATTICE": "test graph", "Jz0": J[0][0], "Jxy0": J[0][1],
         "J1": J[1][0], "Jz2": J[2][0], "Jxy2": J[2][1], "h0": h[0], "h1": h[1], "CONSERVED_QUANTUMNUMBERS": "Sz",
         "NUMBER_EIGENVALUES": 1}
    res = sparsediag.run(p)
    bonds = [(s, d, J[t][0], J[t][1], 0.0) for s, d, t in edges]
    site_h = [h[t] for t in vt]
    assert [s["quantumnumbers"][0][1] for s in res["sectors"]] == [str(k) for k in range(-5, 6)]
    for s, n_up in zip(res["sectors"], range(0, n + 1)):
        w = np.linalg.eigvalsh(oracle.Matrix(n, n_up, bonds, site_h=site_h).dense())
        assert abs(s["energies"][0] - w[0]) < 1e-10, n_up


def test_measurements_on_a_graph(tmp_path):
    """MEASURE_AVERAGE / _LOCAL / _CORRELATIONS on a <GRAPH> (one distance class per ordered vertex pair) equal the
    oracle's operator expectations in the dense ground state (1e-8)."""
    from oracle import measure as omeasure
    n = 8
    edges = [(i, (i + 1) % n) for i in range(n)] + [(0, 4), (1, 6)]
    vt = [i % 3 for i in range(n)]
    hs = {0: 0.07, 1: -0.05, 2: 0.11}
    xml = ['<LATTICES>', f'<GRAPH name="ring+" vertices="{n}">']
    xml += [f'  <VERTEX id="{i + 1}" type="{t}"/>' for i, t in enumerate(vt)]
    xml += [f'  <EDGE source="{s + 1}" target="{d + 1}"/>' for s, d in edges]
    xml += ['</GRAPH>', '</LATTICES>']
    f = tmp_path / "g.xml"
    f.write_text("\n".join(xml))
    meas = {"MEASURE_AVERAGE[M]": "Sz", "MEASURE_LOCAL[Local]": "Sz", "MEASURE_CORRELATIONS[ZZ]": "Sz",
            "MEASURE_CORRELATIONS[PM]": "Splus:Sminus", "MEASURE_CORRELATIONS[MP]": "Sminus:Splus"}
    p = {"MODEL": "spin", "LATTICE_LIBRARY": str(f), "LATTICE": "ring+", "J": 1, "h0": hs[0], "h1": hs[1],
         "h2": hs[2], "CONSERVED_QUANTUMNUMBERS": "Sz", "Sz_total": 1, "NUMBER_EIGENVALUES": 1, **meas}
    res = sparsediag.run(p)
    got = res["sectors"][0]["measurements"][0]
    bonds = [(s, d, 1.0, 1.0, 0.0) for s, d in edges]
    M = oracle.Matrix(n, 5, bonds, site_h=[hs[t] for t in vt])
    w, Z = np.linalg.eigh(M.dense())
    assert abs(w[0] - res["sectors"][0]["energies"][0]) < 1e-9 and w[1] - w[0] > 1e-6
    st, psi = M.states(), Z[:, 0]
    ex = lambda ops: omeasure._expect(st, psi, n, ops)
    assert abs(got["average"]["M"] - sum(ex([("Sz", i)]) for i in range(n)) / n) < 1e-8
    np.testing.assert_allclose(got["local"]["Local"], [ex([("Sz", i)]) for i in range(n)], atol=1e-8)
    for name, (a, b) in (("ZZ", ("Sz", "Sz")), ("PM", ("Splus", "Sminus")), ("MP", ("Sminus", "Splus"))):
        ref = [ex([(a, i), (b, j)]) for i in range(n) for j in range(n)]
        np.testing.assert_allclose(got["correlations"][name], ref, atol=1e-8)
