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
