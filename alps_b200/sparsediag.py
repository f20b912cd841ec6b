"""The sparsediag task around the engine: the loop over Sz sectors and the results.

Reference paths are relative to the ALPS source tree.

`run(params)` follows DiagMatrix::dostep (applications/diag/diag.h:85-137) for
the Sz-conserved spin models the engine handles (local_S = 1/2 .. 2): when
`Sz_total` is not given, every Sz_total from -N S to N S (step 1; diag.h:142-175 takes the range
from the site bases) is a sector, each solved by SparseDiagMatrix::do_subspace
(here `Hamiltonian.solve`, NUMBER_EIGENVALUES / MAX_ITERATIONS from the
parameters); a fixed `Sz_total` gives one sector without quantum-number labels,
as in the reference.  With translation symmetry (TRANSLATION_SYMMETRY, default
true, on a lattice with periodic directions) each Sz sector splits into its
momentum sectors, the momentum loop innermost, labelled TOTAL_MOMENTUM =
write_vector(k) (diag.h:93-131); a given TOTAL_MOMENTUM fixes one momentum and
adds no label.  The ground-state energy and the gap are chosen as in
SparseDiagMatrix::write_xml_body (sparsediag.h:59-90), and `write_xml` writes
the EIGENVALUES and AVERAGES elements of DiagTask::write_xml_body
(src/alps/scheduler/diag.hpp:127-140) and sparsediag.h:80-88.  (The HDF5
archive, diag.hpp:112-124, needs h5py, which this image lacks.)
"""

from __future__ import annotations

import re
from fractions import Fraction
from xml.sax.saxutils import escape

import numpy as np

from . import AEDError, FP64, Hamiltonian, lattice_momenta, lattice_translations, model_from_parameters, momentum_label
from . import measure as _measure


def half_integer_text(v: Fraction) -> str:
    """alps::half_integer printing (src/alps/model/half_integer.h:243-253): "3", "-1/2"."""
    twice = int(2 * v)
    return str(twice // 2) if twice % 2 == 0 else f"{twice}/2"


_VALUE_CHARS = set("#'()*+-./^_")


def parameter_list(text: str) -> list:
    """The tasks of an ALPS parameter file (alps::ParameterList::parse, src/alps/parameter/parameterlist.C:16-40
    with the grammars of parameterlist_p.h:35-47, parameters_p.h:19-26 and parameter_p.h:22-41): `key=value`
    assignments separated by ';', ',' or line ends set global values; a `{ ... }` block is one task, the
    globals at that point plus its own assignments (an empty block: the globals alone); `#clear` drops the
    globals, `#stop` ends the list; blanks and // and /* */ comments are skipped.  Keys start with a letter
    and continue with letters, digits, _ ' # or a [...] suffix; values are "..." or '...' or a run of
    letters, digits and # ' ( ) * + - . / ^ _.  Returns one dict of string values per task."""
    s = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    s = re.sub(r"//[^\n]*", "", s)
    n, i = len(s), 0
    glob, tasks = {}, []

    def err(msg):
        line = s.count("\n", 0, i) + 1
        raise AEDError(-1, f"parameter list, line {line}: {msg}")

    def skip(eol):
        nonlocal i
        while i < n and (s[i] in " \t\r" or (eol and s[i] == "\n")):
            i += 1

    def assignment(target):
        nonlocal i
        j = i
        if not s[i].isalpha():
            err(f"a parameter name expected at {s[i:i + 20]!r}")
        i += 1
        while i < n and (s[i].isalnum() or s[i] in "_'#" or s[i] == "["):
            if s[i] == "[":
                k = s.find("]", i)
                if k < 0:
                    err("unterminated [ in a parameter name")
                i = k
            i += 1
        key = s[j:i]
        skip(False)
        if i >= n or s[i] != "=":
            err(f"'=' expected after {key}")
        i += 1
        skip(False)
        if i < n and s[i] in "\"'":
            k = s.find(s[i], i + 1)
            if k < 0:
                err(f"unterminated string for {key}")
            val, i = s[i + 1:k], k + 1
        else:
            j = i
            while i < n and (s[i].isalnum() or s[i] in _VALUE_CHARS or s.startswith("${", i)):
                if s.startswith("${", i):
                    k = s.find("}", i)
                    if k < 0:
                        err("unterminated ${")
                    i = k
                i += 1
            val = s[j:i]
        target[key] = val
        skip(False)
        if i < n and s[i] in ";,":
            i += 1

    while True:
        skip(True)
        if i >= n:
            break
        if s.startswith("#stop", i):
            break
        if s.startswith("#clear", i):
            glob.clear()
            i += len("#clear")
            skip(False)
            if i < n and s[i] == ";":
                i += 1
            continue
        if s[i] == "{":
            i += 1
            local = dict(glob)
            while True:
                skip(True)
                if i >= n:
                    err("unterminated {")
                if s[i] == "}":
                    i += 1
                    break
                assignment(local)
            tasks.append(local)
            continue
        assignment(glob)
    return tasks


def run_list(text: str, precision=FP64, device=0, seed=0) -> list:
    """run() for every task of a parameter file (parameter_list): [(task parameters, result)]."""
    return [(p, run(p, precision=precision, device=device, seed=seed)) for p in parameter_list(text)]


def _site_info(params: dict):
    """(number of sites, 2 S) of the model (the parser needs a compatible Sz_total: 0 or 1/2)."""
    for trial in (0, 0.5):
        try:
            m = model_from_parameters(dict(params, Sz_total=trial))
            return m["n_sites"], m["two_s"]
        except AEDError:
            continue
    raise AEDError(-1, "cannot read the lattice from the parameters")


def sz_sectors(params: dict) -> list:
    """The Sz_total values of the sector loop: [None] (one unlabelled sector) when Sz_total is given or Sz is
    not conserved, else -N S .. N S in steps of 1 (diag.h:142-175)."""
    qns = str(params.get("CONSERVED_QUANTUMNUMBERS", "")).replace(",", " ").split()
    if "Sz_total" in params or "Sz" not in qns:
        return [None]
    n, two_s = _site_info(params)
    return [Fraction(k, 2) for k in range(-n * two_s, n * two_s + 1, 2)]


def run(params: dict, precision=FP64, device=0, seed=0, workers=1) -> dict:
    """Eigenvalues of every sector: {"sectors": [{"quantumnumbers": [(name, value)], "energies": array,
    "dimension": D, "iterations": m}], "ground_state_energy": E0, "energy_gap": gap}.  Momentum sectors
    run in FP64 whatever `precision` says.  workers > 1 solves that many sectors at once (each on its own
    handle and stream, host threads; the sectors are independent, so the results and their order are those
    of the one-by-one loop)."""
    params = dict(params)
    momenta = lattice_momenta(params)
    req = _measure.requests(params)
    measuring = any(req.values())
    geometry = _measure.Geometry(params) if measuring else None
    label_k = bool(momenta) and not str(params.get("TOTAL_MOMENTUM", "")).strip()
    jobs = []
    for sz in sz_sectors(params):
        p = params if sz is None else dict(params, Sz_total=float(sz))
        mp = model_from_parameters(p)
        for k in momenta or [None]:
            jobs.append((sz, p, mp, k))

    def solve_sector(job):
        sz, p, mp, k = job
        qn = [] if sz is None else [("Sz", half_integer_text(sz))]
        if k is None:
            ham = Hamiltonian.from_parameters(p, precision=precision, device=device)
        else:
            if label_k:
                qn.append(("TOTAL_MOMENTUM", momentum_label(k)))
            ham = Hamiltonian(mp["n_sites"], mp["n_up"], mp["bonds"], FP64, device, mp["site_h"], mp["site_d"],
                              translations=lattice_translations(params, k), two_s=mp["two_s"])
        try:
            if ham.dim == 0:  # empty sector: skipped, as dostep does (diag.h:114)
                return None
            r = ham.solve(nev=max(1, mp["nev"]), max_iter=mp["max_iter"], seed=seed)
            sec = {"quantumnumbers": qn, "energies": np.array(r["evals"]), "dimension": ham.dim,
                   "iterations": r["iterations"], "converged": r["converged"]}
            if measuring and len(r["evals"]):
                # perform_measurements on every eigenvector (diag.h:191-314, sparsediag.h:151-159)
                vecs, _, _ = ham.eigenvectors(k=len(r["evals"]), seed=seed)
                sec["measurements"] = [_measure.measure(ham, v, params, geometry) for v in vecs]
                for v in vecs:
                    v.free()
            return sec
        finally:
            ham.close()

    if workers > 1 and len(jobs) > 1:
        from concurrent.futures import ThreadPoolExecutor

        with ThreadPoolExecutor(max_workers=workers) as pool:
            done = list(pool.map(solve_sector, jobs))
    else:
        done = [solve_sector(j) for j in jobs]
    sectors = [sec for sec in done if sec is not None]
    e0, gap = ground_state_and_gap([s["energies"] for s in sectors])
    return {"sectors": sectors, "ground_state_energy": e0, "energy_gap": gap}


def ground_state_and_gap(energies):
    """(ground-state energy, gap) over sectors as SparseDiagMatrix::write_xml_body picks them
    (sparsediag.h:62-76): the lowest value, and the next one among each sector's lowest (and the
    second of the sector holding the minimum when it is found); None where undefined."""
    inf = float("inf")
    min_val = exc_val = inf
    for ev in energies:
        ev = np.asarray(ev)
        if ev.size >= 1:
            if ev[0] < min_val:
                exc_val = min_val
                min_val = float(ev[0])
                if ev.size >= 2 and ev[1] < exc_val:
                    exc_val = float(ev[1])
            elif ev[0] < exc_val:
                exc_val = float(ev[0])
    return (None if min_val == inf else min_val), (None if exc_val == inf else exc_val - min_val)


def _num(v) -> str:
    """A number as oxstream writes it (boost::lexical_cast<std::string>(double): 17 significant digits)."""
    return "%.17g" % float(v)


def _coord(c) -> str:
    """alps::coordinate_to_string (src/alps/lattice/coordinate_traits.h:97-110), default precision."""
    return "( " + ",".join("%g" % float(x) for x in c) + " )"


def _labels(params):
    """Site, distance and momentum labels of the lattice (graph_helper::site_labels,
    hypercubic_lattice::distance_labels / momenta_labels, hypercubic.h:291-314)."""
    g = _measure.Geometry(params)
    sites = [_coord(c) for c in g.coords]
    dist = [""] * g.num_distances()
    for i in range(g.n):
        for j in range(g.n):
            d = g.distance(i, j)
            if not dist[d]:  # a graph: the vertex numbers (graph_helper::distance_labels, graph_helper.h:535-553)
                dist[d] = f"{i} -- {j}" if g.graph else _coord(g.coords[i]) + " -- " + _coord(g.coords[j])
    moms = [] if g.graph else [_coord(k) for k in g.momenta()]
    return sites, dist, moms


def write_xml(result: dict, path: str, params: dict | None = None) -> None:
    """The spectrum and the eigenstate measurements in the reference's XML elements: AVERAGES with the
    ground-state energy and gap (sparsediag.h:78-88), EIGENVALUES per sector, and EIGENSTATES per sector
    with each eigenstate's measurements, "Energy" included (DiagTask::write_xml_body,
    src/alps/scheduler/diag.hpp:127-160; EigenvectorMeasurements::write_xml_one_vector,
    src/alps/scheduler/measurement_operators.h:209-266: averages, local values, correlations and
    structure factors, each group in name order, indexed by site, distance and momentum labels)."""
    params = params or {}
    lines = ["<?xml version=\"1.0\" encoding=\"UTF-8\"?>", "<SIMULATION>"]
    if params:
        lines.append("  <PARAMETERS>")
        for k, v in params.items():
            lines.append(f"    <PARAMETER name=\"{escape(str(k))}\">{escape(str(v))}</PARAMETER>")
        lines.append("  </PARAMETERS>")
    lines.append("  <AVERAGES>")
    if result["ground_state_energy"] is not None:
        lines.append("    <SCALAR_AVERAGE name=\"Ground State Energy\"><MEAN>"
                     f"{_num(result['ground_state_energy'])}</MEAN></SCALAR_AVERAGE>")
    if result["energy_gap"] is not None:
        lines.append(f"    <SCALAR_AVERAGE name=\"Energy Gap\"><MEAN>{_num(result['energy_gap'])}</MEAN></SCALAR_AVERAGE>")
    lines.append("  </AVERAGES>")

    def qn_lines(s):
        return [f"    <QUANTUMNUMBER name=\"{escape(name)}\" value=\"{escape(value)}\"/>"
                for name, value in s["quantumnumbers"]]

    for s in result["sectors"]:
        ev = s["energies"]
        lines.append(f"  <EIGENVALUES number=\"{ev.size}\">")
        lines += qn_lines(s)
        lines += [_num(e) for e in ev]
        lines.append("  </EIGENVALUES>")
    measuring = any(_measure.requests(params).values())
    if measuring or str(params.get("MEASURE_ENERGY", "true")).lower() not in ("false", "0"):
        labels = _labels(params) if measuring else None
        for s in result["sectors"]:
            ev = s["energies"]
            lines.append(f"  <EIGENSTATES number=\"{ev.size}\">")
            lines += qn_lines(s)
            for j in range(ev.size):
                lines.append(f"    <EIGENSTATE number=\"{j}\">")
                m = s["measurements"][j] if "measurements" in s else {}
                avg = dict(m.get("average", {}), Energy=float(ev[j]))
                for name in sorted(avg):
                    lines.append(f"      <SCALAR_AVERAGE name=\"{escape(name)}\"><MEAN>{_num(avg[name])}</MEAN>"
                                 "</SCALAR_AVERAGE>")
                for group, lab in (("local", 0), ("correlations", 1), ("structure_factor", 2)):
                    for name in sorted(m.get(group, {})):
                        lines.append(f"      <VECTOR_AVERAGE name=\"{escape(name)}\">")
                        for idx, v in zip(labels[lab], m[group][name]):
                            lines.append(f"        <SCALAR_AVERAGE indexvalue=\"{escape(idx)}\"><MEAN>{_num(v)}</MEAN>"
                                         "</SCALAR_AVERAGE>")
                        lines.append("      </VECTOR_AVERAGE>")
                lines.append("    </EIGENSTATE>")
            lines.append("  </EIGENSTATES>")
    lines.append("</SIMULATION>")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
