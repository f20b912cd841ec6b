"""B200 exact-diagonalisation engine for the ALPS sparsediag Lanczos path.

Python face of libaed.so (C ABI in include/aed.h).  The engine keeps ALPS's
parameter surface (LATTICE, MODEL, J/J1, CONSERVED_QUANTUMNUMBERS, Sz_total,
NUMBER_EIGENVALUES) and the ietl vector-space / mult() operations; every call
goes to the CUDA library.  There is no CPU fallback: importing the engine
without a built libaed.so raises, and calls without a GPU fail with the
library's error message.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = [
    "AEDError", "Hamiltonian", "DeviceVector", "Server", "parse_parameters", "model_from_parameters", "lib",
    "FP64", "FP32",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libaed.so")

FP64 = 0
FP32 = 1
MAX_NEV = 16
# aed_solve_result.refined_by: how a mixed solve's FP32 values were refined
REFINED_BY = {0: "none", 1: "rayleigh_ritz", 2: "lanczos"}
MAX_BONDS = 128

OK = 0
ERR_INVALID = -1
ERR_NOMEM = -2
ERR_ADMISSION = -3
ERR_CUDA = -4
ERR_TIMEOUT = -5
ERR_NOT_CONVERGED = -6
ERR_TRIDIAG = -7
ERR_MISMATCH = -8
ERR_CANCELLED = -9
PENDING = 1


class AEDError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"aed error {code}: {msg}")
        self.code = code


class ModelDesc(ctypes.Structure):
    _fields_ = [
        ("n_sites", ctypes.c_int32), ("n_up", ctypes.c_int32), ("n_bonds", ctypes.c_int32),
        ("bond_s1", ctypes.POINTER(ctypes.c_int32)), ("bond_s2", ctypes.POINTER(ctypes.c_int32)),
        ("bond_jz", ctypes.POINTER(ctypes.c_double)), ("bond_jxy", ctypes.POINTER(ctypes.c_double)),
        ("bond_k", ctypes.POINTER(ctypes.c_double)), ("site_h", ctypes.POINTER(ctypes.c_double)),
        ("site_d", ctypes.POINTER(ctypes.c_double)),
    ]


class Translations(ctypes.Structure):
    _fields_ = [("n_trans", ctypes.c_int32), ("site_map", ctypes.POINTER(ctypes.c_int32)),
                ("phase", ctypes.POINTER(ctypes.c_double))]


class ParamInfo(ctypes.Structure):
    _fields_ = [
        ("n_sites", ctypes.c_int32), ("n_up", ctypes.c_int32), ("n_bonds", ctypes.c_int32),
        ("number_eigenvalues", ctypes.c_int32), ("max_iterations", ctypes.c_int32),
        ("has_site_terms", ctypes.c_int32), ("two_s", ctypes.c_int32),
    ]


class SolveOpts(ctypes.Structure):
    _fields_ = [
        ("nev", ctypes.c_int32), ("max_iter", ctypes.c_int32), ("rtol", ctypes.c_double),
        ("atol", ctypes.c_double), ("seed", ctypes.c_uint64), ("start", ctypes.POINTER(ctypes.c_double)),
        ("refine", ctypes.c_int32), ("profile", ctypes.c_int32), ("resume", ctypes.c_int32),
        ("reorth", ctypes.c_int32),
    ]


class SolveResult(ctypes.Structure):
    _fields_ = [
        ("n_evals", ctypes.c_int32), ("iterations", ctypes.c_int32), ("iterations_low", ctypes.c_int32),
        ("converged", ctypes.c_int32), ("evals", ctypes.c_double * MAX_NEV),
        ("errors", ctypes.c_double * MAX_NEV), ("evals_low", ctypes.c_double * MAX_NEV),
        ("seconds", ctypes.c_double), ("apply_ms", ctypes.c_double), ("refined_by", ctypes.c_int32),
    ]


class ServerOpts(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32), ("max_slots", ctypes.c_int32), ("steps_per_launch", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("hbm_fraction", ctypes.c_double), ("hbm_budget_bytes", ctypes.c_int64),
        ("reserve_bytes", ctypes.c_int64), ("max_lanes", ctypes.c_int32), ("lane_min_dim", ctypes.c_int64),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("resident", ctypes.c_int32), ("queued", ctypes.c_int32), ("bytes_used", ctypes.c_int64),
        ("bytes_budget", ctypes.c_int64), ("graph_launches", ctypes.c_int64), ("lanes", ctypes.c_int32),
    ]


_lib = None
_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_I32P = ctypes.POINTER(ctypes.c_int32)
_I64P = ctypes.POINTER(ctypes.c_int64)
_U32P = ctypes.POINTER(ctypes.c_uint32)


def lib():
    """The loaded libaed.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libaed.so not found at {LIB_PATH}: run `python -m alps_b200.build` "
                              "(the engine has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "aed_last_error": (ctypes.c_char_p, []),
            "aed_parse_parameters": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ParamInfo), _I32P, _I32P, _DP,
                                                    _DP, _DP, _DP, _DP, _I32, _I32]),
            "aed_parse_graph_parameters": (ctypes.c_int, [ctypes.c_char_p, _I32, _I32P, _I32, _I32P, _I32P, _I32P,
                                                          ctypes.POINTER(ParamInfo), _I32P, _I32P, _DP, _DP, _DP,
                                                          _DP, _DP, _I32, _I32]),
            "aed_create": (ctypes.c_int, [ctypes.POINTER(ModelDesc), ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(_P)]),
            "aed_destroy": (ctypes.c_int, [_P]),
            "aed_empty_cache": (ctypes.c_int, [ctypes.c_int]),
            "aed_reserve_basis": (ctypes.c_int, [_P, _I32]),
            "aed_create_momentum": (ctypes.c_int, [ctypes.POINTER(ModelDesc), ctypes.POINTER(Translations),
                                                   ctypes.c_int, ctypes.POINTER(_P)]),
            "aed_momentum_basis": (ctypes.c_int, [_P, _U32P, _DP, _I64, _I64]),
            "aed_create_spin": (ctypes.c_int, [ctypes.POINTER(ModelDesc), ctypes.c_int32, ctypes.c_int,
                                               ctypes.POINTER(_P)]),
            "aed_spin_basis": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64), _I64, _I64]),
            "aed_create_spin_momentum": (ctypes.c_int, [ctypes.POINTER(ModelDesc), ctypes.c_int32,
                                                        ctypes.POINTER(Translations), ctypes.c_int,
                                                        ctypes.POINTER(_P)]),
            "aed_expectation": (ctypes.c_int, [_P, _P, ctypes.c_int32, _I32, _I32P, _I32P, _DP]),
            "aed_momentum_expectation": (ctypes.c_int, [_P, _P, ctypes.c_int32, _I32, _I32P, _I32P, _DP]),
            "aed_lattice_geometry": (ctypes.c_int, [ctypes.c_char_p, _I32P, _I32P, _I32P]),
            "aed_lattice_momenta": (ctypes.c_int, [ctypes.c_char_p, _I32P, _I32P, _DP, _I32]),
            "aed_lattice_translations": (ctypes.c_int, [ctypes.c_char_p, _DP, _I32, _I32P, _I32P, _I32P, _DP, _I32]),
            "aed_set_couplings": (ctypes.c_int, [_P, ctypes.POINTER(ModelDesc)]),
            "aed_dimension": (ctypes.c_int, [_P, _I64P]),
            "aed_basis_copy": (ctypes.c_int, [_P, _U32P, _I64, _I64]),
            "aed_basis_state": (ctypes.c_int, [_P, _I64, ctypes.POINTER(ctypes.c_uint64)]),
            "aed_index": (ctypes.c_int, [_P, _U32P, _I64, _I64P]),
            "aed_vec_alloc": (ctypes.c_int, [_P, ctypes.POINTER(_P)]),
            "aed_vec_free": (ctypes.c_int, [_P, _P]),
            "aed_vec_upload": (ctypes.c_int, [_P, _P, _DP]),
            "aed_vec_download": (ctypes.c_int, [_P, _P, _DP]),
            "aed_vec_copy": (ctypes.c_int, [_P, _P, _P]),
            "aed_vec_clear": (ctypes.c_int, [_P, _P]),
            "aed_vec_fill_random": (ctypes.c_int, [_P, _P, ctypes.c_uint64]),
            "aed_mult": (ctypes.c_int, [_P, _P, _P]),
            "aed_dot": (ctypes.c_int, [_P, _P, _P, _DP]),
            "aed_nrm2": (ctypes.c_int, [_P, _P, _DP]),
            "aed_axpy": (ctypes.c_int, [_P, _D, _P, _P]),
            "aed_scal": (ctypes.c_int, [_P, _D, _P]),
            "aed_div": (ctypes.c_int, [_P, _D, _P]),
            "aed_lanczos_step": (ctypes.c_int, [_P, _P, _P, _P, _D, _DP, _DP]),
            "aed_solve": (ctypes.c_int, [_P, ctypes.POINTER(SolveOpts), ctypes.POINTER(SolveResult)]),
            "aed_last_tmatrix": (ctypes.c_int, [_P, _DP, _DP, _I32, _I32P]),
            "aed_eigenvectors": (ctypes.c_int, [_P, ctypes.POINTER(SolveOpts), _I32, ctypes.POINTER(_P), _DP, _DP]),
            "aed_lanczos_state_bytes": (ctypes.c_int, [_P, _I64P]),
            "aed_lanczos_save": (ctypes.c_int, [_P, ctypes.c_void_p, _I64]),
            "aed_lanczos_load": (ctypes.c_int, [_P, ctypes.c_char_p, _I64]),
            "aed_time_mult": (ctypes.c_int, [_P, _P, _P, _I32, _DP]),
            "aed_time_apply": (ctypes.c_int, [_P, _P, _P, _I32, _I32, _I32, _DP, _I32P]),
            "aed_apply_variant_count": (_I32, []),
            "aed_apply_variant_name": (ctypes.c_char_p, [_I32]),
            "aed_get_stream": (ctypes.c_int, [_P, ctypes.POINTER(_P)]),
            "aed_lanczos_vector": (ctypes.c_int, [_P, ctypes.c_int32, _P]),
            "aed_last_tmatrix_fp32": (ctypes.c_int, [_P, _DP, _DP, _I32, _I32P]),
            "aed_launch_count": (ctypes.c_int, [_I64P]),
            "aed_dot_noalloc": (ctypes.c_int, [_P, _P, _I64, ctypes.c_int, _P, _P]),
            "aed_tmatrix": (ctypes.c_int, [_I32, _DP, _DP, _I32, _DP, _DP, _I32P, _I32P]),
            "aed_server_create": (ctypes.c_int, [ctypes.POINTER(ServerOpts), ctypes.POINTER(_P)]),
            "aed_server_destroy": (ctypes.c_int, [_P]),
            "aed_server_submit": (ctypes.c_int, [_P, ctypes.POINTER(ModelDesc), ctypes.POINTER(SolveOpts), _I64P]),
            "aed_server_step": (ctypes.c_int, [_P, _I32P]),
            "aed_server_poll": (ctypes.c_int, [_P, _I64, ctypes.POINTER(SolveResult)]),
            "aed_server_cancel": (ctypes.c_int, [_P, _I64]),
            "aed_server_get_stats": (ctypes.c_int, [_P, ctypes.POINTER(ServerStats)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc not in (OK, PENDING):
        msg = lib().aed_last_error()
        raise AEDError(rc, msg.decode() if msg else "")
    return rc


def _dp(a):
    return a.ctypes.data_as(_DP) if a is not None else None


def tmatrix(alpha, beta):
    """The engine's Tmatrix::compute(true): distinct non-ghost values, errors, multiplicities."""
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    b = np.ascontiguousarray(beta, dtype=np.float64)
    n = a.size
    ev, er = np.zeros(max(n, 1)), np.zeros(max(n, 1))
    mu = np.zeros(max(n, 1), np.int32)
    cnt = ctypes.c_int32(0)
    _check(lib().aed_tmatrix(n, _dp(a), _dp(b), n, _dp(ev), _dp(er), mu.ctypes.data_as(_I32P), ctypes.byref(cnt)))
    c = cnt.value
    return {"evals": ev[:c], "errors": er[:c], "mults": mu[:c]}


def apply_variants() -> list:
    """Names of the apply variants (index = the `variant` of Hamiltonian.time_apply)."""
    L = lib()
    return [L.aed_apply_variant_name(v).decode() for v in range(L.aed_apply_variant_count())]


def empty_cache(device: int = 0) -> None:
    """Give the memory cached from destroyed handles back to the driver (aed_empty_cache)."""
    _check(lib().aed_empty_cache(device))


def launch_count() -> int:
    """Engine kernel launches made by this process so far."""
    c = ctypes.c_int64(0)
    _check(lib().aed_launch_count(ctypes.byref(c)))
    return c.value


def _parsed_model(call):
    """Run a parse entry point twice (counts, then arrays) and return its model dict; call(info, arrays...)
    takes the ParamInfo and the seven output arrays with their capacities."""
    info = ParamInfo()
    _check(call(ctypes.byref(info), None, None, None, None, None, None, None, 0, 0))
    nb, ns = info.n_bonds, info.n_sites
    s1, s2 = np.zeros(max(nb, 1), np.int32), np.zeros(max(nb, 1), np.int32)
    jz, jxy, kq = np.zeros(max(nb, 1)), np.zeros(max(nb, 1)), np.zeros(max(nb, 1))
    sh, sd = np.zeros(ns), np.zeros(ns)
    _check(call(ctypes.byref(info), s1.ctypes.data_as(_I32P), s2.ctypes.data_as(_I32P), _dp(jz), _dp(jxy), _dp(kq),
                _dp(sh), _dp(sd), nb, ns))
    bonds = [(int(s1[b]), int(s2[b]), float(jz[b]), float(jxy[b]), float(kq[b])) for b in range(nb)]
    return {"n_sites": ns, "n_up": info.n_up, "bonds": bonds, "nev": info.number_eigenvalues,
            "max_iter": info.max_iterations, "two_s": info.two_s,
            "site_h": sh if info.has_site_terms else None, "site_d": sd if info.has_site_terms else None}


def parse_parameters(text: str):
    """ALPS parameter text -> dict(n_sites, n_up, bonds=[(s1, s2, Jz, Jxy, K)], nev, max_iter, two_s, site_h,
    site_d)."""
    t = text.encode()
    return _parsed_model(lambda *a: lib().aed_parse_parameters(t, *a))


class Graph(tuple):
    """(n, vertex types, edges [(source, target, type)]) with the vertices' coordinates (empty lists where
    the file gives none) as .coords."""

    def __new__(cls, n, vtype, edges, coords):
        g = super().__new__(cls, (n, vtype, edges))
        g.coords = coords
        return g


def read_graph(path: str, name: str):
    """<GRAPH name="..."> of a lattice library file (read_graph_xml, src/alps/lattice/graph.h:121-222):
    a Graph (number of vertices, vertex types, edges [(source, target, type)] in file order; vertex
    COORDINATEs as .coords), vertices numbered from 0; None when the file holds no graph of that name.  A
    VERTEX without id takes the next number of its own counter, types default to 0, and an edge to a vertex
    beyond the list adds it."""
    import xml.etree.ElementTree as ET
    root = ET.parse(path).getroot()
    for g in ([root] if root.tag == "GRAPH" else root.iter("GRAPH")):
        if g.get("name") != name:
            continue
        fixed = bool(g.get("vertices"))
        vtype = [0] * (int(g.get("vertices")) if fixed else 0)
        counter, edges, coords = 0, [], {}
        for el in g:
            if el.tag == "VERTEX":
                if el.get("id"):
                    vid = int(el.get("id")) - 1
                else:
                    vid, counter = counter, counter + 1
                if vid >= len(vtype):
                    if fixed:
                        raise AEDError(ERR_INVALID, f"graph {name!r}: too many vertices in <GRAPH>")
                    vtype += [0] * (vid + 1 - len(vtype))
                vtype[vid] = int(el.get("type") or 0)
                c = el.find("COORDINATE")
                if c is not None and (c.text or "").strip():
                    coords[vid] = [float(v) for v in c.text.replace(",", " ").split()]
            elif el.tag == "EDGE":
                edges.append((int(el.get("source")) - 1, int(el.get("target")) - 1, int(el.get("type") or 0)))
            else:
                raise AEDError(ERR_INVALID, f"graph {name!r}: illegal element <{el.tag}> in <GRAPH>")
        n = max([len(vtype)] + [max(a, b) + 1 for a, b, _ in edges])
        return Graph(n, vtype + [0] * (n - len(vtype)), edges, [coords.get(i, []) for i in range(n)])
    return None


def graph_of(params):
    """The <GRAPH> a parameter dict names (graph_helper::make_graph, src/alps/lattice/graph_helper.h:653-684):
    GRAPH, or a LATTICE that LATTICE_LIBRARY holds as a <GRAPH>; None for the built-in lattices (no
    LATTICE_LIBRARY: the reference's own lattices.xml, which the engine restates).  As LatticeLibrary
    (src/alps/lattice/latticelibrary.C:25-74) a LATTICE_LIBRARY that is missing or not well-formed is an
    error, and so is a name the library does not hold; a <LATTICEGRAPH> of a library is not read by this
    engine and is refused rather than replaced by a built-in lattice of the same name."""
    if not isinstance(params, dict):
        return None
    has_g, has_l = "GRAPH" in params, "LATTICE" in params
    if has_g and has_l:
        raise AEDError(ERR_INVALID, "both GRAPH and LATTICE were specified")
    name = str(params.get("GRAPH", params.get("LATTICE", ""))).strip().strip('"')
    lib_path = str(params.get("LATTICE_LIBRARY", "")).strip().strip('"')
    if not lib_path:
        if has_g:
            raise AEDError(ERR_INVALID, f"GRAPH {name!r} not found (LATTICE_LIBRARY must name the file holding it)")
        return None
    if not os.path.isfile(lib_path):
        raise AEDError(ERR_INVALID, f"Could not find lattice library file {lib_path!r} (LATTICE_LIBRARY)")
    import xml.etree.ElementTree as ET
    try:
        g = read_graph(lib_path, name)
        if g is not None:
            return g
        root = ET.parse(lib_path).getroot()
    except ET.ParseError as e:
        raise AEDError(ERR_INVALID, f"LATTICE_LIBRARY {lib_path!r}: {e}") from None
    if any(el.get("name") == name for el in root.iter("LATTICEGRAPH")):
        raise AEDError(ERR_INVALID, f"lattice {name!r} of LATTICE_LIBRARY {lib_path!r} is a <LATTICEGRAPH>: only "
                                    "<GRAPH> elements of a lattice library are supported")
    raise AEDError(ERR_INVALID, f"{'GRAPH' if has_g else 'LATTICE'} {name!r} not found in LATTICE_LIBRARY "
                                f"{lib_path!r}")


def parse_graph_parameters(text: str, graph):
    """parse_parameters for a graph (n, vertex types, edges) instead of a built-in lattice
    (aed_parse_graph_parameters)."""
    n, vtype, edges = graph
    vt = np.ascontiguousarray(vtype, dtype=np.int32)
    es = np.ascontiguousarray([e[0] for e in edges] or [0], dtype=np.int32)
    et = np.ascontiguousarray([e[1] for e in edges] or [0], dtype=np.int32)
    ey = np.ascontiguousarray([e[2] for e in edges] or [0], dtype=np.int32)
    t = text.encode()
    return _parsed_model(lambda *a: lib().aed_parse_graph_parameters(
        t, n, vt.ctypes.data_as(_I32P), len(edges), es.ctypes.data_as(_I32P), et.ctypes.data_as(_I32P),
        ey.ctypes.data_as(_I32P), *a))


def _params_text(params) -> str:
    if isinstance(params, dict):
        lines = []
        for k, v in params.items():
            if isinstance(v, str) and not v.replace(".", "", 1).replace("-", "", 1).isdigit():
                lines.append(f'{k} = "{v}"')
            else:
                lines.append(f"{k} = {v}")
        return "\n".join(lines)
    return params


def model_from_parameters(params) -> dict:
    """dict or text of ALPS parameters -> parse_parameters() result (a dict naming a <GRAPH>: its bonds)."""
    g = graph_of(params)
    if g is not None:
        return parse_graph_parameters(_params_text(params), g)
    return parse_parameters(_params_text(params))


def lattice_momenta(params) -> list:
    """Momenta of the sparsediag sector loop (aed_lattice_momenta): TOTAL_MOMENTUM when given, else every
    translation momentum when TRANSLATION_SYMMETRY (default true), else [].  A <GRAPH> has no translations."""
    if graph_of(params) is not None:
        if str(params.get("TOTAL_MOMENTUM", "")).strip():
            raise AEDError(ERR_INVALID, "TOTAL_MOMENTUM on a GRAPH: a graph has no translations")
        return []
    txt = _params_text(params).encode()
    n, nd = ctypes.c_int32(0), ctypes.c_int32(0)
    _check(lib().aed_lattice_momenta(txt, ctypes.byref(n), ctypes.byref(nd), None, 0))
    k = np.zeros(max(n.value * nd.value, 1))
    _check(lib().aed_lattice_momenta(txt, ctypes.byref(n), ctypes.byref(nd), _dp(k), n.value))
    return [tuple(k[m * nd.value:(m + 1) * nd.value]) for m in range(n.value)]


def lattice_translations(params, k) -> list:
    """[(phase, site map)] of the lattice at momentum k (aed_lattice_translations), the identity first."""
    txt = _params_text(params).encode()
    kk = np.ascontiguousarray(k, dtype=np.float64).reshape(-1)
    nt, ns = ctypes.c_int32(0), ctypes.c_int32(0)
    _check(lib().aed_lattice_translations(txt, _dp(kk), kk.size, ctypes.byref(nt), ctypes.byref(ns), None, None, 0))
    mp = np.zeros(max(nt.value * ns.value, 1), np.int32)
    ph = np.zeros(max(2 * nt.value, 1))
    _check(lib().aed_lattice_translations(txt, _dp(kk), kk.size, ctypes.byref(nt), ctypes.byref(ns),
                                          mp.ctypes.data_as(_I32P), _dp(ph), nt.value))
    return [(complex(ph[2 * t], ph[2 * t + 1]), [int(v) for v in mp[t * ns.value:(t + 1) * ns.value]])
            for t in range(nt.value)]


def momentum_label(k) -> str:
    """The TOTAL_MOMENTUM value of a sector: alps::write_vector(k), 20 significant digits."""
    return " ".join("%.20g" % v for v in k)


class DeviceVector:
    """A device vector of the handle's precision (ietl vector_type)."""

    def __init__(self, ham: "Hamiltonian"):
        self.ham = ham
        p = _P()
        _check(lib().aed_vec_alloc(ham._h, ctypes.byref(p)))
        self.ptr = p

    def free(self):
        if self.ptr is not None and self.ptr.value:
            lib().aed_vec_free(self.ham._h, self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            if self.ham._h:
                self.free()
        except Exception:
            pass

    def upload(self, host):
        host = self.ham._host_vector(host)
        _check(lib().aed_vec_upload(self.ham._h, self.ptr, _dp(host)))
        return self

    def download(self):
        out = np.empty(self.ham.vlen)
        _check(lib().aed_vec_download(self.ham._h, self.ptr, _dp(out)))
        return out.view(np.complex128) if self.ham.momentum else out


class Hamiltonian:
    """One Sz sector of a spin model on one GPU (an aed_handle; local spin two_s / 2, spin 1/2 on the
    bit-exact engine unless `generic`); with `translations` (a list of (phase, site map), the identity
    first, as lattice_translations returns) one momentum sector of it, whose vectors are complex."""

    def __init__(self, n_sites, n_up, bonds, precision=FP64, device=0, site_h=None, site_d=None, translations=None,
                 two_s=1, generic=False):
        self.n_sites, self.n_up = int(n_sites), int(n_up)
        self.bonds = [tuple(b) for b in bonds]
        self.precision = precision
        nb = len(self.bonds)
        self._s1 = np.array([b[0] for b in self.bonds] or [0], np.int32)
        self._s2 = np.array([b[1] for b in self.bonds] or [0], np.int32)
        self._jz = np.array([b[2] for b in self.bonds] or [0.0])
        self._jxy = np.array([b[3] for b in self.bonds] or [0.0])
        self._k = np.array([(b[4] if len(b) > 4 else 0.0) for b in self.bonds] or [0.0])
        self._sh = None if site_h is None else np.ascontiguousarray(site_h, dtype=np.float64)
        self._sd = None if site_d is None else np.ascontiguousarray(site_d, dtype=np.float64)
        desc = ModelDesc(self.n_sites, self.n_up, nb, self._s1.ctypes.data_as(_I32P), self._s2.ctypes.data_as(_I32P),
                         _dp(self._jz), _dp(self._jxy), _dp(self._k), _dp(self._sh), _dp(self._sd))
        h = _P()
        self._h = None
        self.momentum = translations is not None
        self.two_s = int(two_s)
        self.spin_s = self.two_s != 1 or generic  # the spin-S engine (aed_create_spin)
        if self.momentum:
            if precision != FP64:
                raise AEDError(ERR_INVALID, "momentum sectors are FP64")
            self._tmap = np.ascontiguousarray([m for _, m in translations], dtype=np.int32).reshape(-1)
            self._tph = np.ascontiguousarray([[p.real, p.imag] for p, _ in translations], dtype=np.float64)
            tr = Translations(len(translations), self._tmap.ctypes.data_as(_I32P), _dp(self._tph))
            if self.spin_s:
                _check(lib().aed_create_spin_momentum(ctypes.byref(desc), self.two_s, ctypes.byref(tr), device,
                                                      ctypes.byref(h)))
            else:
                _check(lib().aed_create_momentum(ctypes.byref(desc), ctypes.byref(tr), device, ctypes.byref(h)))
        elif self.spin_s:
            if precision != FP64:
                raise AEDError(ERR_INVALID, "spin-S sectors are FP64")
            _check(lib().aed_create_spin(ctypes.byref(desc), self.two_s, device, ctypes.byref(h)))
        else:
            _check(lib().aed_create(ctypes.byref(desc), precision, device, ctypes.byref(h)))
        self._h = h
        d = ctypes.c_int64(0)
        _check(lib().aed_dimension(self._h, ctypes.byref(d)))
        self.dim = d.value
        self.vlen = 2 * self.dim if self.momentum else self.dim

    def _host_vector(self, v):
        """A host vector as the engine's layout: float64, interleaved (re, im) in a momentum sector."""
        if self.momentum:
            v = np.ascontiguousarray(v, dtype=np.complex128).view(np.float64)
        else:
            v = np.ascontiguousarray(v, dtype=np.float64)
        if v.size != self.vlen:
            raise AEDError(ERR_INVALID, f"vector of {v.size} values, the sector needs {self.vlen}")
        return v

    def set_couplings(self, bonds, site_h=None, site_d=None):
        """Re-target this handle to a new bond list on the same sector."""
        nb = len(bonds)
        self.bonds = [tuple(b) for b in bonds]
        self._s1 = np.array([b[0] for b in self.bonds] or [0], np.int32)
        self._s2 = np.array([b[1] for b in self.bonds] or [0], np.int32)
        self._jz = np.array([b[2] for b in self.bonds] or [0.0])
        self._jxy = np.array([b[3] for b in self.bonds] or [0.0])
        self._k = np.array([(b[4] if len(b) > 4 else 0.0) for b in self.bonds] or [0.0])
        self._sh = None if site_h is None else np.ascontiguousarray(site_h, dtype=np.float64)
        self._sd = None if site_d is None else np.ascontiguousarray(site_d, dtype=np.float64)
        desc = ModelDesc(self.n_sites, self.n_up, nb, self._s1.ctypes.data_as(_I32P), self._s2.ctypes.data_as(_I32P),
                         _dp(self._jz), _dp(self._jxy), _dp(self._k), _dp(self._sh), _dp(self._sd))
        _check(lib().aed_set_couplings(self._h, ctypes.byref(desc)))

    @classmethod
    def from_parameters(cls, params, precision=FP64, device=0):
        """The sector a parameter set names: its Sz_total, and its TOTAL_MOMENTUM when translation
        symmetry is on (a set that loops over momenta needs TOTAL_MOMENTUM or TRANSLATION_SYMMETRY=false:
        alps_b200.sparsediag runs the loops)."""
        m = model_from_parameters(params)
        ks = lattice_momenta(params)
        trans = None
        if ks:
            if len(ks) > 1:
                raise AEDError(ERR_INVALID, "the parameters loop over momenta: give TOTAL_MOMENTUM (one sector per "
                                            "handle; alps_b200.sparsediag loops over them) or TRANSLATION_SYMMETRY=false")
            trans = lattice_translations(params, ks[0])
        ham = cls(m["n_sites"], m["n_up"], m["bonds"], precision, device, m["site_h"], m["site_d"], translations=trans,
                  two_s=m["two_s"])
        ham.params = m
        ham.total_momentum = ks[0] if ks else None
        return ham

    def momentum_basis(self):
        """(representative states, normalisations) of a momentum sector (aed_momentum_basis; a spin-S
        sector's representatives are 64-bit packed digits, from aed_spin_basis)."""
        nm = np.empty(self.dim)
        if self.spin_s:
            st = self.basis()
            _check(lib().aed_momentum_basis(self._h, None, _dp(nm), 0, self.dim))
            return st, nm
        st = np.empty(self.dim, np.uint32)
        _check(lib().aed_momentum_basis(self._h, st.ctypes.data_as(_U32P), _dp(nm), 0, self.dim))
        return st, nm

    def close(self):
        if self._h:
            lib().aed_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- basis ---------------------------------------------------------------
    def basis(self, offset=0, count=None):
        count = self.dim - offset if count is None else count
        if self.spin_s:  # packed digits, 64-bit (aed_spin_basis)
            out = np.empty(count, np.uint64)
            _check(lib().aed_spin_basis(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), offset, count))
            return out
        out = np.empty(count, np.uint32)
        _check(lib().aed_basis_copy(self._h, out.ctypes.data_as(_U32P), offset, count))
        return out

    def state(self, idx: int) -> int:
        """The state of row idx (aed_basis_state): bit string, representative or packed digits."""
        out = ctypes.c_uint64(0)
        _check(lib().aed_basis_state(self._h, int(idx), ctypes.byref(out)))
        return out.value

    def index(self, states):
        st = np.ascontiguousarray(states, dtype=np.uint32)
        out = np.empty(st.size, np.int64)
        _check(lib().aed_index(self._h, st.ctypes.data_as(_U32P), st.size, out.ctypes.data_as(_I64P)))
        return out

    # -- ietl vector space ------------------------------------------------------
    def new_vector(self):
        return DeviceVector(self)

    def mult(self, x: DeviceVector, y: DeviceVector):
        _check(lib().aed_mult(self._h, x.ptr, y.ptr))

    def apply(self, xh):
        """Host convenience: y = H x for a host vector (uploads, applies, downloads)."""
        x = self.new_vector().upload(xh)
        y = self.new_vector()
        self.mult(x, y)
        out = y.download()
        x.free()
        y.free()
        return out

    def dot(self, x, y):
        out = ctypes.c_double(0)
        _check(lib().aed_dot(self._h, x.ptr, y.ptr, ctypes.byref(out)))
        return out.value

    def two_norm(self, x):
        out = ctypes.c_double(0)
        _check(lib().aed_nrm2(self._h, x.ptr, ctypes.byref(out)))
        return out.value

    def axpy(self, a, x, y):
        _check(lib().aed_axpy(self._h, a, x.ptr, y.ptr))

    def scal(self, a, x):
        _check(lib().aed_scal(self._h, a, x.ptr))

    def div(self, a, x):
        _check(lib().aed_div(self._h, a, x.ptr))

    def fill_random(self, x, seed):
        _check(lib().aed_vec_fill_random(self._h, x.ptr, seed))

    def copy(self, x, y):
        _check(lib().aed_vec_copy(self._h, x.ptr, y.ptr))

    def lanczos_step(self, v_prev, v_cur, v_next, beta_prev):
        a = ctypes.c_double(0)
        b = ctypes.c_double(0)
        _check(lib().aed_lanczos_step(self._h, v_prev.ptr if v_prev is not None else None, v_cur.ptr, v_next.ptr,
                                      beta_prev, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def time_apply(self, x, y, reps=5, variant=-1, with_alpha=False):
        """(mean ms, variant) of the apply, optionally with the fused step's <x,y> partials."""
        ms = ctypes.c_double(0)
        v = ctypes.c_int32(0)
        _check(lib().aed_time_apply(self._h, x.ptr, y.ptr, reps, variant, 1 if with_alpha else 0, ctypes.byref(ms),
                                    ctypes.byref(v)))
        return ms.value, v.value

    def reserve_basis(self, vectors):
        """Allocate the FP32 Lanczos basis store of a mixed-precision handle for `vectors` vectors now
        (aed_reserve_basis), so that no later solve grows it."""
        _check(lib().aed_reserve_basis(self._h, int(vectors)))

    def time_mult(self, x, y, reps=10):
        ms = ctypes.c_double(0)
        _check(lib().aed_time_mult(self._h, x.ptr, y.ptr, reps, ctypes.byref(ms)))
        return ms.value

    # -- solves ---------------------------------------------------------------------
    def solve(self, nev=1, max_iter=0, seed=0, start=None, rtol=0.0, atol=0.0, refine=0, profile=False,
              resume=False, reorth=False):
        """Lanczos eigenvalues (aed_solve).  resume=True continues the live FP64 recurrence (the last
        solve's, or one restored by lanczos_load) until nev values converge.  reorth=True (FP32 handles)
        reorthogonalises every FP32 Lanczos vector against the stored basis."""
        st = None if start is None else self._host_vector(start)
        opts = SolveOpts(nev, max_iter, rtol, atol, seed, _dp(st), refine, 1 if profile else 0, 1 if resume else 0,
                         1 if reorth else 0)
        res = SolveResult()
        _check(lib().aed_solve(self._h, ctypes.byref(opts), ctypes.byref(res)))
        n = res.n_evals
        return {"evals": np.array(res.evals[:n]), "errors": np.array(res.errors[:n]),
                "iterations": res.iterations, "iterations_low": res.iterations_low,
                "evals_low": np.array(res.evals_low[:n]), "converged": bool(res.converged),
                "seconds": res.seconds, "apply_ms": res.apply_ms, "refined_by": REFINED_BY[res.refined_by]}

    def eigenvectors(self, k=1, seed=0, start=None):
        """Ritz vectors of the k lowest eigenvalues of the last solve (aed_eigenvectors): the solve's
        seed / start must be given again.  Returns (vectors, evals, residuals)."""
        st = None if start is None else self._host_vector(start)
        opts = SolveOpts(k, 0, 0.0, 0.0, seed, _dp(st), 0, 0, 0)
        vecs = [self.new_vector() for _ in range(k)]
        arr = (_P * k)(*[v.ptr for v in vecs])
        ev = np.zeros(k)
        rs = np.zeros(k)
        _check(lib().aed_eigenvectors(self._h, ctypes.byref(opts), k, arr, _dp(ev), _dp(rs)))
        return vecs, ev, rs

    def lanczos_save(self) -> bytes:
        """Checkpoint of the live FP64 recurrence (aed_lanczos_save)."""
        n = ctypes.c_int64(0)
        _check(lib().aed_lanczos_state_bytes(self._h, ctypes.byref(n)))
        if n.value == 0:
            raise AEDError(ERR_INVALID, "no live Lanczos recurrence")
        buf = ctypes.create_string_buffer(n.value)
        _check(lib().aed_lanczos_save(self._h, buf, n.value))
        return buf.raw

    def lanczos_load(self, state: bytes):
        """Restore a checkpoint into this handle (aed_lanczos_load); solve(resume=True) continues it."""
        _check(lib().aed_lanczos_load(self._h, state, len(state)))

    def stream(self) -> int:
        """The handle's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        p = _P()
        _check(lib().aed_get_stream(self._h, ctypes.byref(p)))
        return p.value or 0

    def lanczos_vector(self, j):
        """v_j of the FP32 Lanczos basis the last mixed solve stored (aed_lanczos_vector), as float64."""
        v = self.new_vector()
        _check(lib().aed_lanczos_vector(self._h, j, v.ptr))
        out = v.download()
        v.free()
        return out

    def last_tmatrix(self, fp32_phase=False):
        """alpha, beta of the last solve's FP64 recurrence (aed_last_tmatrix), or with fp32_phase=True of the
        last mixed solve's FP32 phase (aed_last_tmatrix_fp32)."""
        f = lib().aed_last_tmatrix_fp32 if fp32_phase else lib().aed_last_tmatrix
        n = ctypes.c_int32(0)
        _check(f(self._h, None, None, 0, ctypes.byref(n)))
        a = np.zeros(max(n.value, 1))
        b = np.zeros(max(n.value, 1))
        _check(f(self._h, _dp(a), _dp(b), n.value, ctypes.byref(n)))
        return a[: n.value], b[: n.value]


def _result_dict(res):
    n = res.n_evals
    return {"evals": np.array(res.evals[:n]), "errors": np.array(res.errors[:n]), "iterations": res.iterations,
            "iterations_low": res.iterations_low, "evals_low": np.array(res.evals_low[:n]),
            "converged": bool(res.converged), "seconds": res.seconds,
            "refined_by": REFINED_BY.get(res.refined_by, str(res.refined_by))}


class Server:
    """Batched / served Lanczos solves on one GPU (aed_server_*): requests are
    admitted by HBM footprint and advance together, S Lanczos steps per CUDA
    graph launch; new requests join at the next step."""

    def __init__(self, precision=FP32, device=0, max_slots=512, steps=8, hbm_fraction=0.0, hbm_budget=0,
                 reserve=0, max_lanes=0, lane_min_dim=0):
        """reserve: bytes of device memory to map into the server's pool up front (-1: the whole budget).
        Requests of dimension >= lane_min_dim (0: 2^21; -1: none) run as single-instance solves beside the
        batch, max_lanes (0: 2) at once."""
        o = ServerOpts(device, max_slots, steps, precision, hbm_fraction, hbm_budget, reserve, max_lanes, lane_min_dim)
        h = _P()
        self._h = None
        _check(lib().aed_server_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.precision = precision

    def close(self):
        if self._h:
            lib().aed_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, n_sites, n_up, bonds, nev=1, seed=0, max_iter=0, site_h=None, site_d=None):
        nb = len(bonds)
        s1 = np.array([b[0] for b in bonds] or [0], np.int32)
        s2 = np.array([b[1] for b in bonds] or [0], np.int32)
        jz = np.array([b[2] for b in bonds] or [0.0])
        jxy = np.array([b[3] for b in bonds] or [0.0])
        kq = np.array([(b[4] if len(b) > 4 else 0.0) for b in bonds] or [0.0])
        sh = None if site_h is None else np.ascontiguousarray(site_h, dtype=np.float64)
        sd = None if site_d is None else np.ascontiguousarray(site_d, dtype=np.float64)
        desc = ModelDesc(n_sites, n_up, nb, s1.ctypes.data_as(_I32P), s2.ctypes.data_as(_I32P), _dp(jz), _dp(jxy),
                         _dp(kq), _dp(sh), _dp(sd))
        opts = SolveOpts(nev, max_iter, 0.0, 0.0, seed, None, 0, 0)
        t = ctypes.c_int64(0)
        _check(lib().aed_server_submit(self._h, ctypes.byref(desc), ctypes.byref(opts), ctypes.byref(t)))
        return t.value

    def step(self):
        n = ctypes.c_int32(0)
        _check(lib().aed_server_step(self._h, ctypes.byref(n)))
        return n.value

    def poll(self, ticket):
        res = SolveResult()
        rc = lib().aed_server_poll(self._h, ticket, ctypes.byref(res))
        if rc == PENDING:
            return None
        _check(rc)
        return _result_dict(res)

    def cancel(self, ticket):
        _check(lib().aed_server_cancel(self._h, ticket))

    def stats(self):
        st = ServerStats()
        _check(lib().aed_server_get_stats(self._h, ctypes.byref(st)))
        return {"resident": st.resident, "queued": st.queued, "bytes_used": st.bytes_used,
                "bytes_budget": st.bytes_budget, "graph_launches": st.graph_launches, "lanes": st.lanes}

    def run(self, tickets, max_steps=100000):
        """Step until every ticket finished; returns {ticket: result}."""
        out, left = {}, set(tickets)
        for _ in range(max_steps):
            if not left:
                break
            self.step()
            for t in list(left):
                r = self.poll(t)
                if r is not None:
                    out[t] = r
                    left.discard(t)
        if left:
            raise AEDError(ERR_NOT_CONVERGED, f"{len(left)} requests unfinished after {max_steps} steps")
        return out
