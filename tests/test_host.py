"""Host-side checks of libaed.so without a GPU: exports, parameter surface, error paths."""

import ctypes
import json
import os
import re

import numpy as np
import pytest

import alps_b200 as ed
from oracle import bloch
import oracle
from oracle import lattice

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s+(aed_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = ed.lib()
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_apply_variant_names():
    names = ed.apply_variants()
    assert len(names) >= 12 and len(set(names)) == len(names)
    assert ed.lib().aed_apply_variant_name(len(names)) is None
    assert ed.lib().aed_apply_variant_name(-1) is None


PARAM_CASES = [
    {"LATTICE": "chain lattice", "L": 16, "J": 1},
    {"LATTICE": "open chain lattice", "L": 10, "J": 0.7},
    {"LATTICE": "nnn chain lattice", "L": 28, "J": 1, "J1": 0.31},
    {"LATTICE": "nnn open chain lattice", "L": 10, "J": 1, "J1": 0.5},
    {"LATTICE": "square lattice", "L": 6, "W": 5, "J": 1},
    {"LATTICE": "square lattice", "L": 4, "J": 1.5},
    {"LATTICE": "open square lattice", "L": 3, "W": 4, "J": 1.0},
    {"LATTICE": "anisotropic square lattice", "L": 10, "W": 3, "J0": 1, "J1": 0.4},
    {"LATTICE": "ladder", "L": 12, "J0": 1.2, "J1": 0.8},
    {"LATTICE": "open ladder", "L": 6, "J0": 1, "J1": 2},
    {"LATTICE": "chain lattice", "L": 2, "J": 1},
    {"LATTICE": "nnn chain lattice", "L": 4, "J": 1, "J1": 1},
    {"LATTICE": "chain lattice", "L": 8, "Jz": 1.3, "Jxy": 0.6},
    {"LATTICE": "nnn chain lattice", "L": 8, "J": 1, "Jz1": 0.2, "Jxy1": 0.9},
]


@pytest.mark.parametrize("p", PARAM_CASES)
def test_parameter_surface_matches_oracle(p):
    p = dict(p, MODEL="spin", CONSERVED_QUANTUMNUMBERS="Sz", Sz_total=0, TRANSLATION_SYMMETRY="false")
    m = ed.model_from_parameters(p)
    N, nu, bonds = lattice.spin_model(p)
    assert m["n_sites"] == N and m["n_up"] == nu
    assert len(m["bonds"]) == len(bonds)
    for a, b in zip(m["bonds"], bonds):
        assert a[0] == b[0] and a[1] == b[1]
        assert a[2] == pytest.approx(b[2], abs=0) and a[3] == pytest.approx(b[3], abs=0)


def test_parameter_surface_matches_golden_example6():
    """The reference's example6 (anisotropic square 10x4) has 40 sites, beyond the
    engine's 32; the oracle lattice is pinned to it (tests/test_oracle.py) and the
    engine is checked against the oracle on 10x3 with the same edge rules."""
    with open(os.path.join(ROOT, "tests", "golden", "lattice_example6.json")) as f:
        g = json.load(f)
    _, _, ob = lattice.lattice_graph("anisotropic square lattice", {"L": 10, "W": 4})
    assert [list(b) for b in ob] == g["bonds"]
    txt = ('MODEL="spin"\nLATTICE="anisotropic square lattice"\nL=10\nW=3\nJ0=1\nJ1=2\n'
           'CONSERVED_QUANTUMNUMBERS="Sz"\nSz_total=0\nTRANSLATION_SYMMETRY=false\n')
    m = ed.parse_parameters(txt)
    _, _, ob3 = lattice.lattice_graph("anisotropic square lattice", {"L": 10, "W": 3})
    assert [[b[0], b[1]] for b in m["bonds"]] == [[s, t] for s, t, _ in ob3]
    # J per bond type: type 0 -> J0, type 1 -> J1
    assert [b[2] for b in m["bonds"]] == [1.0 if t == 0 else 2.0 for _, _, t in ob3]


def test_parameter_file_syntax_and_defaults():
    txt = """// sparsediag job
    MODEL = "spin"; LATTICE = "nnn chain lattice"
    L = 2*7, J = 1
    J1 = 1/4
    local_S = 1/2
    CONSERVED_QUANTUMNUMBERS = "Sz"
    Sz_total = 1
    TRANSLATION_SYMMETRY = false
    NUMBER_EIGENVALUES = 3
    MAX_ITERATIONS = 200
    h = 0.1
    """
    m = ed.parse_parameters(txt)
    assert m["n_sites"] == 14 and m["n_up"] == 8
    assert m["nev"] == 3 and m["max_iter"] == 200
    assert m["bonds"][1][2] == 0.25 and m["bonds"][0][2] == 1.0
    assert np.allclose(m["site_h"], 0.1)


@pytest.mark.parametrize("bad,msg", [
    ('MODEL="spin"\nLATTICE="chain lattice"\nL=8\nTRANSLATION_SYMMETRY=false\nCONSERVED_QUANTUMNUMBERS="Sz"\n',
     "Sz_total"),
    ('MODEL="boson Hubbard"\nLATTICE="chain lattice"\nL=8\n', "MODEL"),
    ('MODEL="spin"\nLATTICE="kagome lattice"\nL=8\n', "LATTICE"),
    ('MODEL="spin"\nLATTICE="chain lattice"\nL=8\nlocal_S=5/2\n', "local_S"),
    ('MODEL="spin"\nLATTICE="chain lattice"\nL=40\nSz_total=0\nCONSERVED_QUANTUMNUMBERS="Sz"\n'
     'TRANSLATION_SYMMETRY=false\n', "sites"),
    ('MODEL="spin"\nLATTICE="chain lattice"\nL=8\nSz_total=0\nCONSERVED_QUANTUMNUMBERS="Sz"\n'
     'TRANSLATION_SYMMETRY=false\nJ="0.8+0.4*random()"\n', "random"),
    ('MODEL="spin"\nLATTICE="chain lattice"\nL=8\nCONSERVED_QUANTUMNUMBERS="N"\n', "Sz"),
])
def test_parameter_errors(bad, msg):
    with pytest.raises(ed.AEDError) as e:
        ed.parse_parameters(bad)
    assert e.value.code == ed.ERR_INVALID
    assert msg in str(e.value)


def test_create_reports_invalid_models_before_touching_a_device():
    with pytest.raises(ed.AEDError) as e:
        ed.Hamiltonian(40, 20, [])
    assert e.value.code in (ed.ERR_INVALID, ed.ERR_CUDA)
    with pytest.raises(ed.AEDError):
        ed.Hamiltonian(4, 2, [(0, 0, 1.0, 1.0)])


def test_create_without_gpu_fails_loudly():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    with pytest.raises(ed.AEDError) as e:
        ed.Hamiltonian(4, 2, [(0, 1, 1.0, 1.0), (1, 2, 1.0, 1.0)])
    assert e.value.code == ed.ERR_CUDA


@pytest.mark.parametrize("L,nev,seed", [(12, 4, 1), (14, 4, 11), (14, 2, 3)])
def test_engine_tmatrix_matches_oracle_and_lapack(L, nev, seed):
    """The engine's T-matrix analysis (shared by the host driver and the batched
    device check) against the oracle's and the LAPACK-based restatement."""
    N, nu, bonds = lattice.spin_model({"LATTICE": "chain lattice", "L": L, "J": 1, "Sz_total": 0})
    r = oracle.Matrix(N, nu, bonds).lanczos(nev=nev, seed=seed)
    a, b = r["alpha"], r["beta"]
    for m in sorted({2, 3, 7, 20, len(a) // 2, len(a)}):
        t = ed.tmatrix(a[:m], b[:m])
        o = oracle.tmatrix(a[:m], b[:m])
        lp = oracle.tmatrix_lapack(a[:m], b[:m])
        assert len(t["evals"]) == len(o["evals"]) == len(lp["evals"])
        np.testing.assert_allclose(t["evals"], lp["evals"], rtol=1e-12, atol=1e-12)
        assert list(t["mults"]) == list(lp["mults"])
        # error estimates are |beta z_last|; below ~eps*|T| they are rounding noise
        np.testing.assert_allclose(t["errors"], lp["errors"], rtol=1e-5, atol=1e-13)


def test_sparsediag_gap_rule_and_labels(tmp_path):
    """The ground state / gap choice of sparsediag.h:62-76 and the half-integer labels."""
    from fractions import Fraction
    import xml.etree.ElementTree as ET

    from alps_b200 import sparsediag

    e0, gap = sparsediag.ground_state_and_gap([[-1.0, -0.5], [-2.0, -1.2], [-1.5]])
    assert e0 == -2.0 and gap == pytest.approx(0.5)  # -1.5 (another sector) lies below -1.2
    e0, gap = sparsediag.ground_state_and_gap([[-2.0, -1.9], [-1.0]])
    assert gap == pytest.approx(0.1)
    assert sparsediag.ground_state_and_gap([[-3.0]]) == (-3.0, None)
    assert [sparsediag.half_integer_text(Fraction(k, 2)) for k in (-3, -2, 0, 1, 4)] == ["-3/2", "-1", "0", "1/2", "2"]
    res = {"sectors": [{"quantumnumbers": [("Sz", "1/2")], "energies": np.array([-1.25, -0.75])}],
           "ground_state_energy": -1.25, "energy_gap": 0.5}
    sparsediag.write_xml(res, str(tmp_path / "s.xml"), {"LATTICE": "chain lattice", "L": 5})
    root = ET.parse(tmp_path / "s.xml").getroot()
    ev = root.find("EIGENVALUES")
    assert ev.get("number") == "2" and ev.find("QUANTUMNUMBER").get("value") == "1/2"
    text = (ev.text or "") + "".join(c.tail or "" for c in ev)
    assert [float(v) for v in text.split()] == [-1.25, -0.75]


MOMENTUM_CASES = [
    ("chain lattice", {"L": 8}), ("nnn chain lattice", {"L": 7}), ("square lattice", {"L": 3, "W": 4}),
    ("anisotropic square lattice", {"L": 4, "W": 2}), ("ladder", {"L": 5}), ("open chain lattice", {"L": 6}),
    ("open ladder", {"L": 4}),
]


@pytest.mark.parametrize("lat,geo", MOMENTUM_CASES, ids=[c[0] for c in MOMENTUM_CASES])
def test_lattice_momenta_and_translations_match_oracle(lat, geo):
    """The engine's translation momenta and translations (site maps, phases) equal the oracle's restatement of
    hypercubic_lattice (pinned by the example13-15 fixtures)."""
    p = dict(geo, MODEL="spin", LATTICE=lat, CONSERVED_QUANTUMNUMBERS="Sz", Sz_total=0)
    ks = ed.lattice_momenta(p)
    ref = bloch.translation_momenta(lat, geo)
    assert ks == ref
    for k in ks:
        got = ed.lattice_translations(p, k)
        exp = bloch.translations(lat, geo, k)
        assert [m for _, m in got] == [m for _, m in exp]
        assert all(abs(a - b) <= 1e-15 for (a, _), (b, _) in zip(got, exp))
    assert ed.lattice_momenta(dict(p, TRANSLATION_SYMMETRY="false")) == []
    if ks:
        one = ed.lattice_momenta(dict(p, TOTAL_MOMENTUM=ed.momentum_label(ks[-1])))
        assert one == [ks[-1]]
        assert ed.momentum_label(ks[-1]) == bloch.momentum_label(ks[-1])


def test_total_momentum_needs_one_component_per_periodic_direction():
    with pytest.raises(ed.AEDError, match="TOTAL_MOMENTUM"):
        ed.lattice_momenta('MODEL="spin"\nLATTICE="square lattice"\nL=3\nTOTAL_MOMENTUM="0"\nSz_total=0\n')


def test_sparsediag_xml_eigenstates_with_measurements(tmp_path):
    """write_xml: EIGENVALUES and EIGENSTATES per sector, each eigenstate's SCALAR_AVERAGEs in name order
    with Energy, VECTOR_AVERAGEs indexed by site / distance / momentum labels (DiagTask::write_xml_body,
    write_xml_one_vector), numbers with 17 significant digits."""
    import xml.etree.ElementTree as ET
    from alps_b200 import sparsediag
    p = {"MODEL": "spin", "LATTICE": "square lattice", "L": 2, "W": 3, "J": 1,
         "MEASURE_AVERAGE[Magnetization]": "Sz", "MEASURE_LOCAL[Local magnetization]": "Sz",
         "MEASURE_CORRELATIONS[Diagonal spin correlations]": "Sz",
         "MEASURE_STRUCTURE_FACTOR[Structure Factor S]": "Sz"}
    meas = {"average": {"Magnetization": 0.1}, "local": {"Local magnetization": list(np.arange(6) * 0.5)},
            "correlations": {"Diagonal spin correlations": list(np.arange(6) * 0.25)},
            "structure_factor": {"Structure Factor S": list(np.arange(6) * 1.0)}}
    res = {"ground_state_energy": -1.0, "energy_gap": 0.5,
           "sectors": [{"quantumnumbers": [("Sz", "0")], "energies": np.array([-1.0, 0.1]),
                        "measurements": [meas, meas]}]}
    out = tmp_path / "s.xml"
    sparsediag.write_xml(res, str(out), p)
    root = ET.parse(out).getroot()
    st = root.findall("EIGENSTATES")
    assert len(st) == 1 and st[0].get("number") == "2"
    e1 = st[0].findall("EIGENSTATE")[1]
    assert [a.get("name") for a in e1.findall("SCALAR_AVERAGE")] == ["Energy", "Magnetization"]
    assert e1.findall("SCALAR_AVERAGE")[0].find("MEAN").text == "0.10000000000000001"
    va = {v.get("name"): v for v in e1.findall("VECTOR_AVERAGE")}
    assert [s.get("indexvalue") for s in va["Local magnetization"]] == \
        ["( 0,0 )", "( 0,1 )", "( 0,2 )", "( 1,0 )", "( 1,1 )", "( 1,2 )"]
    assert [s.get("indexvalue") for s in va["Diagonal spin correlations"]][:3] == \
        ["( 0,0 ) -- ( 0,0 )", "( 0,0 ) -- ( 0,1 )", "( 0,0 ) -- ( 0,2 )"]
    assert [s.get("indexvalue") for s in va["Structure Factor S"]][:4] == \
        ["( 0,0 )", "( 0,2.0944 )", "( 0,-2.0944 )", "( 3.14159,0 )"]


def test_local_spin_parameters():
    """local_S = 1: two_s = 2 and the sector's digit sum Sz_total + N S."""
    m = ed.parse_parameters('MODEL="spin"\nLATTICE="chain lattice"\nL=6\nlocal_S=1\nJ=1\n'
                            'CONSERVED_QUANTUMNUMBERS="Sz"\nSz_total=-2\nTRANSLATION_SYMMETRY=false\n')
    assert m["two_s"] == 2 and m["n_up"] == 4
    m = ed.parse_parameters('MODEL="spin"\nLATTICE="chain lattice"\nL=5\nlocal_S=3/2\nJ=1\n'
                            'CONSERVED_QUANTUMNUMBERS="Sz"\nSz_total=1/2\nTRANSLATION_SYMMETRY=false\n')
    assert m["two_s"] == 3 and m["n_up"] == 8


@pytest.mark.parametrize("lat,geo", [("chain lattice", {"L": 6}), ("open chain lattice", {"L": 5}),
                                     ("square lattice", {"L": 3, "W": 4}), ("ladder", {"L": 4}),
                                     ("anisotropic square lattice", {"L": 2, "W": 3})])
def test_measurement_geometry_matches_oracle(lat, geo):
    """Distance classes, their count and the momenta of the measurement code (from the engine's lattice
    geometry) equal the oracle's restatement of hypercubic_lattice."""
    from alps_b200 import measure
    from oracle import measure as om
    p = dict(geo, LATTICE=lat)
    g = measure.Geometry(p)
    ext, per, coords = om._geometry(p)
    assert g.coords == coords and g.num_distances() == om._num_distances(ext, per)
    for i in range(g.n):
        for j in range(g.n):
            assert g.distance(i, j) == om._distance(ext, per, coords[i], coords[j])
    ks = []
    for cc in coords:
        ks.append([2 * np.pi * ((x - L) if x > L // 2 else x) / L for x, L in zip(cc, ext)])
    assert np.allclose(g.momenta(), ks)


def test_spin_momentum_constructor_checks_translations_before_the_device():
    """aed_create_spin_momentum refuses translations that are not permutations of the sites, or that do not
    start with the identity, before it looks for a device; spin-S momentum handles are FP64 only."""
    n = 4
    s1 = np.arange(n, dtype=np.int32)
    s2 = ((np.arange(n) + 1) % n).astype(np.int32)
    j = np.ones(n)
    desc = ed.ModelDesc(n, n, n, s1.ctypes.data_as(ed._I32P), s2.ctypes.data_as(ed._I32P), ed._dp(j), ed._dp(j),
                        None, None, None)
    ph = np.array([1.0, 0.0, 1.0, 0.0])
    h = ed._P()
    for maps, msg in (([0, 1, 2, 3, 1, 1, 2, 3], "permutation"), ([1, 2, 3, 0, 0, 1, 2, 3], "identity")):
        mp = np.array(maps, dtype=np.int32)
        tr = ed.Translations(2, mp.ctypes.data_as(ed._I32P), ed._dp(ph))
        rc = ed.lib().aed_create_spin_momentum(ctypes.byref(desc), 2, ctypes.byref(tr), 0, ctypes.byref(h))
        assert rc == ed.ERR_INVALID
        assert msg in ed.lib().aed_last_error().decode()
    tr = [(1.0 + 0j, [0, 1, 2, 3]), (1.0 + 0j, [1, 2, 3, 0])]
    with pytest.raises(ed.AEDError, match="FP64"):
        ed.Hamiltonian(n, n, [(i, (i + 1) % n, 1.0, 1.0) for i in range(n)], precision=ed.FP32, translations=tr,
                       two_s=2)


def test_parameter_list_tasks():
    """ALPS parameter files: globals, one task per { } block with the globals at that point, separators ; , and
    line ends, quoted values, bracketed and primed keys, comments, #clear and #stop."""
    from alps_b200 import sparsediag
    txt = ('MODEL="spin";\nLATTICE="chain lattice";  // nearest neighbours\nCONSERVED_QUANTUMNUMBERS="Sz";\n'
           'local_S=1;\nJ=1;\nSz_total=0\n{L=4}\n{L=6}\nSz_total=1\n'
           "{ L=4, J'=0.5; MEASURE_AVERAGE[Magnetization]=Sz }\n/* { L=99 } */\n{}\n#clear\n{ L = 3 }\n#stop\n{ L=100 }\n")
    tasks = sparsediag.parameter_list(txt)
    assert [t.get("L") for t in tasks] == ["4", "6", "4", None, "3"]
    assert [t.get("Sz_total") for t in tasks] == ["0", "0", "1", "1", None]
    assert tasks[2]["J'"] == "0.5" and tasks[2]["MEASURE_AVERAGE[Magnetization]"] == "Sz"
    assert tasks[0]["LATTICE"] == "chain lattice" and tasks[4] == {"L": "3"}
    m = ed.model_from_parameters(tasks[1])
    assert (m["n_sites"], m["two_s"], m["n_up"]) == (6, 2, 6)
    m = ed.model_from_parameters(tasks[2])
    assert (m["n_sites"], m["two_s"], m["n_up"]) == (4, 2, 5)
    with pytest.raises(ed.AEDError, match="line 2"):
        sparsediag.parameter_list("L=4\n{ J=1 ")
    with pytest.raises(ed.AEDError, match="'='"):
        sparsediag.parameter_list("L 4")


@pytest.mark.parametrize("local_s,L,expect", [("1/2", 5, [f"{k}/2" for k in range(-5, 6, 2)]),
                                              ("1", 5, [str(k) for k in range(-5, 6)]),
                                              ("3/2", 3, [f"{k}/2" for k in range(-9, 10, 2)]),
                                              ("2", 2, [str(k) for k in range(-4, 5)])])
def test_sz_sector_loop_covers_minus_ns_to_ns(local_s, L, expect):
    """Without Sz_total the loop runs Sz_total = -N S .. N S in steps of 1, odd chains of integer spin included."""
    from alps_b200 import sparsediag
    p = {"MODEL": "spin", "LATTICE": "chain lattice", "L": L, "local_S": local_s, "J": 1,
         "CONSERVED_QUANTUMNUMBERS": "Sz"}
    assert [sparsediag.half_integer_text(v) for v in sparsediag.sz_sectors(p)] == expect
    assert sparsediag.sz_sectors(dict(p, Sz_total=0)) == [None]


GRAPH_XML = """<LATTICES>
<GRAPH name="two dimers" vertices="4">
  <VERTEX id="1" type="0"/>
  <VERTEX id="2" type="0"/>
  <VERTEX id="3" type="1"/>
  <VERTEX id="4" type="1"/>
  <EDGE type="0" source="1" target="2"/>
  <EDGE type="0" source="3" target="4"/>
  <EDGE type="1" source="1" target="3"/>
  <EDGE type="1" source="2" target="4"/>
</GRAPH>
<GRAPH name="grown">
  <VERTEX type="2"/>
  <VERTEX/>
  <EDGE source="1" target="2"/>
  <EDGE source="2" target="5" type="3"/>
</GRAPH>
</LATTICES>
"""


def test_graph_of_a_lattice_library(tmp_path):
    """<GRAPH> lattices: vertices and edges as read_graph_xml reads them, bonds in file order with the couplings
    of their edge type, site terms of their vertex type, no translations; GRAPH and LATTICE are exclusive."""
    f = tmp_path / "graphs.xml"
    f.write_text(GRAPH_XML)
    assert ed.read_graph(str(f), "grown") == (5, [2, 0, 0, 0, 0], [(0, 1, 0), (1, 4, 3)])
    assert ed.read_graph(str(f), "none") is None
    p = {"MODEL": "spin", "LATTICE_LIBRARY": str(f), "LATTICE": "two dimers", "J0": 1, "J1": 0.25, "Jz1": 0.5,
         "h1": 0.3, "D": 0.1, "CONSERVED_QUANTUMNUMBERS": "Sz", "Sz_total": 0}
    m = ed.model_from_parameters(p)
    assert (m["n_sites"], m["n_up"], m["two_s"]) == (4, 2, 1)
    assert m["bonds"] == [(0, 1, 1.0, 1.0, 0.0), (2, 3, 1.0, 1.0, 0.0), (0, 2, 0.5, 0.25, 0.0), (1, 3, 0.5, 0.25, 0.0)]
    assert list(m["site_h"]) == [0.0, 0.0, 0.3, 0.3] and list(m["site_d"]) == [0.1] * 4
    g = dict(p, GRAPH="two dimers")
    del g["LATTICE"]
    assert ed.model_from_parameters(g)["bonds"] == m["bonds"]
    assert ed.lattice_momenta(p) == []
    from alps_b200 import measure, sparsediag
    assert [sparsediag.half_integer_text(v) for v in sparsediag.sz_sectors({k: v for k, v in p.items()
                                                                           if k != "Sz_total"})] == ["-2", "-1", "0",
                                                                                                    "1", "2"]
    with pytest.raises(ed.AEDError, match="both GRAPH and LATTICE"):
        ed.model_from_parameters(dict(p, GRAPH="two dimers"))
    with pytest.raises(ed.AEDError, match="not found"):
        ed.model_from_parameters({k: v for k, v in g.items() if k != "LATTICE_LIBRARY"})
    assert measure.Geometry(p).graph
    with pytest.raises(ed.AEDError, match="translations"):
        ed.lattice_momenta(dict(p, TOTAL_MOMENTUM="0"))
    # a lattice library without that lattice: an error, as LatticeLibrary has it; without a library the
    # built-in lattices
    q = {"MODEL": "spin", "LATTICE_LIBRARY": str(f), "LATTICE": "chain lattice", "L": 4, "J": 1,
         "CONSERVED_QUANTUMNUMBERS": "Sz", "Sz_total": 0}
    with pytest.raises(ed.AEDError, match="not found in LATTICE_LIBRARY"):
        ed.model_from_parameters(q)
    del q["LATTICE_LIBRARY"]
    assert ed.model_from_parameters(q)["n_sites"] == 4


def test_graph_geometry_and_labels(tmp_path):
    """Measurement geometry of a <GRAPH>: one distance class per ordered vertex pair (i N + j, labelled "i -- j"),
    site labels from the vertices' COORDINATEs ("(  )" without), no momenta (structure factors refused)."""
    from alps_b200 import measure, sparsediag
    f = tmp_path / "g.xml"
    f.write_text('<LATTICES><GRAPH name="tri" vertices="3">'
                 '<VERTEX id="1"><COORDINATE>0 0</COORDINATE></VERTEX><VERTEX id="2"><COORDINATE>1 0</COORDINATE>'
                 '</VERTEX><VERTEX id="3"/>'
                 '<EDGE source="1" target="2"/><EDGE source="2" target="3"/><EDGE source="3" target="1"/>'
                 '</GRAPH></LATTICES>')
    p = {"MODEL": "spin", "LATTICE_LIBRARY": str(f), "LATTICE": "tri", "J": 1, "CONSERVED_QUANTUMNUMBERS": "Sz",
         "MEASURE_CORRELATIONS[C]": "Sz"}
    g = measure.Geometry(p)
    assert g.graph and g.n == 3 and g.num_distances() == 9
    assert [g.distance(i, j) for i in range(3) for j in range(3)] == list(range(9))
    sites, dist, moms = sparsediag._labels(p)
    assert sites == ["( 0,0 )", "( 1,0 )", "(  )"]
    assert dist[:4] == ["0 -- 0", "0 -- 1", "0 -- 2", "1 -- 0"] and moms == []
    with pytest.raises(ed.AEDError, match="momenta"):
        g.momenta()


def test_xml_labels_match_the_reference_label_output():
    """Site, bond, momentum and distance labels of the 4x4 square lattice (the index values of the XML
    eigenstate measurements) equal the reference's test/lattice/label.output; the bond labels follow the
    engine's bond list, so they also pin its bond order."""
    from alps_b200 import sparsediag
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "labels_square4.json")))
    p = {"MODEL": "spin", "LATTICE": "square lattice", "L": 4, "J": 1, "CONSERVED_QUANTUMNUMBERS": "Sz",
         "Sz_total": 0}
    sites, dist, moms = sparsediag._labels(p)
    assert sites == g["sites"]
    assert moms == g["momenta"]
    assert dist == g["distances"]
    bonds = ed.model_from_parameters(p)["bonds"]
    assert [f"{sites[a]} -- {sites[b]}" for a, b, *_ in bonds] == g["bonds"]


def test_graph_parameters_refuse_bad_graphs():
    """aed_parse_graph_parameters: an edge joining a vertex to itself, an edge vertex out of range, a negative
    type, too many edges or sites are refused with a message."""
    text = 'MODEL="spin"\nJ=1\nCONSERVED_QUANTUMNUMBERS="Sz"\nSz_total=0\n'.encode()

    def parse(n, edges, vtype=None):
        info = ed.ParamInfo()
        src = np.array([e[0] for e in edges] or [0], np.int32)
        tgt = np.array([e[1] for e in edges] or [0], np.int32)
        typ = np.array([e[2] for e in edges] or [0], np.int32)
        vt = None if vtype is None else np.array(vtype, np.int32).ctypes.data_as(ed._I32P)
        rc = ed.lib().aed_parse_graph_parameters(text, n, vt, len(edges), src.ctypes.data_as(ed._I32P),
                                                 tgt.ctypes.data_as(ed._I32P), typ.ctypes.data_as(ed._I32P),
                                                 ctypes.byref(info), None, None, None, None, None, None, None, 0, 0)
        return rc, ed.lib().aed_last_error().decode(), info

    rc, _, info = parse(4, [(0, 1, 0), (1, 2, 0), (2, 3, 1)])
    assert rc == 0 and (info.n_sites, info.n_bonds, info.n_up) == (4, 3, 2)
    for n, edges, vtype, msg in ((4, [(1, 1, 0)], None, "itself"), (4, [(0, 4, 0)], None, "out of range"),
                                 (4, [(0, 1, -1)], None, "negative edge type"),
                                 (4, [(0, 1, 0)], [0, -2, 0, 0], "negative vertex type"),
                                 (40, [(0, 1, 0)], None, "number of sites"),
                                 (4, [(0, 1, 0)] * 129, None, "too many bonds")):
        rc, err, _ = parse(n, edges, vtype)
        assert rc == ed.ERR_INVALID and msg in err, (msg, err)


def test_lattice_library_errors_as_the_reference(tmp_path):
    """A LATTICE_LIBRARY that is missing or not well-formed is an error (latticelibrary.C:25-39), whether
    GRAPH or LATTICE names the lattice; a library <LATTICEGRAPH> is refused, not replaced by the built-in
    lattice of the same name."""
    f = tmp_path / "broken.xml"
    f.write_text("<LATTICES><GRAPH name='x'>")
    p = {"MODEL": "spin", "LATTICE_LIBRARY": str(f), "LATTICE": "chain lattice", "L": 4, "J": 1,
         "CONSERVED_QUANTUMNUMBERS": "Sz", "Sz_total": 0}
    with pytest.raises(ed.AEDError, match="LATTICE_LIBRARY"):
        ed.model_from_parameters(p)
    with pytest.raises(ed.AEDError, match="LATTICE_LIBRARY"):
        ed.model_from_parameters({k: v for k, v in dict(p, GRAPH="x").items() if k != "LATTICE"})
    with pytest.raises(ed.AEDError, match="Could not find lattice library file"):
        ed.model_from_parameters(dict(p, LATTICE_LIBRARY=str(tmp_path / "missing.xml")))
    g = tmp_path / "latticegraphs.xml"
    g.write_text("<LATTICES><LATTICEGRAPH name='chain lattice'><FINITELATTICE/></LATTICEGRAPH></LATTICES>")
    with pytest.raises(ed.AEDError, match="LATTICEGRAPH"):
        ed.model_from_parameters(dict(p, LATTICE_LIBRARY=str(g)))


def test_bench_seeded_start_equals_the_engines_start_vector():
    """bench.py's end-to-end leg builds the seed-1 start vector on the host: it equals the oracle's
    restatement of the engine's fill_random (pinned to the GPU's bit for bit by the parity tests), across
    the chunk boundary of its generator."""
    import bench

    n = (1 << 22) + 1000
    assert np.array_equal(bench.seeded_start(1, n), oracle.start_vector(1, n))
    assert np.array_equal(bench.seeded_start(7, 5000), oracle.start_vector(7, 5000))
