"""Oracle for the ALPS sparsediag Lanczos path -- CPU restatement, TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this package, and only as the checker (or the timed CPU baseline).  The
engine (alps_b200) never imports it.

The heavy parts live in ed_oracle.cpp (built by ``make -C oracle`` into
libedoracle.so); this module wraps them with ctypes and adds a numpy/scipy
restatement of the ietl Lanczos driver that uses LAPACK's own dstev (scipy), to
pin the C++ tridiagonal solver against LAPACK.  See ed_oracle.cpp for the
reference file:line list.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from . import lattice  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libedoracle.so")
_lib = None

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_dbl_p = ctypes.POINTER(ctypes.c_double)
_c_u32_p = ctypes.POINTER(ctypes.c_uint32)
_c_i64_p = ctypes.POINTER(ctypes.c_int64)
_c_i32_p = ctypes.POINTER(ctypes.c_int32)


def build(force: bool = False) -> str:
    """Compile ed_oracle.cpp in place (g++, OpenMP)."""
    src = os.path.join(_HERE, "ed_oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_basis_build.restype = ctypes.c_int64
        L.orc_basis_build.argtypes = [ctypes.c_int, ctypes.c_int, _c_u32_p, ctypes.c_int64]
        L.orc_index.restype = ctypes.c_int64
        L.orc_index.argtypes = [_c_u32_p, ctypes.c_int64, ctypes.c_uint32]
        L.orc_start_vector.restype = None
        L.orc_start_vector.argtypes = [ctypes.c_uint64, ctypes.c_int64, _c_dbl_p]
        L.orc_matrix_build.restype = ctypes.c_void_p
        L.orc_matrix_build.argtypes = [ctypes.c_int, ctypes.c_int, _c_dbl_p, _c_dbl_p, ctypes.c_int,
                                       _c_int_p, _c_int_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]
        L.orc_matrix_dim.restype = ctypes.c_int64
        L.orc_matrix_dim.argtypes = [ctypes.c_void_p]
        L.orc_matrix_nnz.restype = ctypes.c_int64
        L.orc_matrix_nnz.argtypes = [ctypes.c_void_p]
        L.orc_matrix_states.restype = None
        L.orc_matrix_states.argtypes = [ctypes.c_void_p, _c_u32_p]
        L.orc_matrix_csr.restype = None
        L.orc_matrix_csr.argtypes = [ctypes.c_void_p, _c_i64_p, _c_i32_p, _c_dbl_p]
        L.orc_matrix_mult.restype = None
        L.orc_matrix_mult.argtypes = [ctypes.c_void_p, _c_dbl_p, _c_dbl_p]
        L.orc_matrix_mult_rows.restype = None
        L.orc_matrix_mult_rows.argtypes = [ctypes.c_void_p, _c_dbl_p, _c_dbl_p, ctypes.c_int64, ctypes.c_int64]
        L.orc_matrix_free.restype = None
        L.orc_matrix_free.argtypes = [ctypes.c_void_p]
        L.orc_stev.restype = ctypes.c_int
        L.orc_stev.argtypes = [ctypes.c_int, _c_dbl_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, _c_dbl_p]
        L.orc_tmatrix.restype = ctypes.c_int
        L.orc_tmatrix.argtypes = [ctypes.c_int, _c_dbl_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, _c_int_p,
                                  ctypes.c_int, _c_dbl_p, _c_dbl_p]
        L.orc_lanczos.restype = ctypes.c_int
        L.orc_lanczos.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint64, _c_dbl_p,
                                  ctypes.c_double, ctypes.c_double, _c_dbl_p, _c_dbl_p, _c_int_p, _c_int_p,
                                  _c_dbl_p, _c_dbl_p, ctypes.c_int]
        L.orc_hv_matfree.restype = None
        L.orc_hv_matfree.argtypes = [ctypes.c_int, _c_u32_p, ctypes.c_int64, ctypes.c_int, _c_int_p, _c_int_p,
                                     _c_dbl_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, ctypes.c_int64, ctypes.c_int64]
        L.orc_basis_fast.restype = ctypes.c_int64
        L.orc_basis_fast.argtypes = [ctypes.c_int, ctypes.c_int, _c_u32_p, ctypes.c_int64]
        L.orc_sample_times.restype = None
        L.orc_sample_times.argtypes = [ctypes.c_int, _c_u32_p, ctypes.c_int64, ctypes.c_int, _c_int_p, _c_int_p,
                                       _c_dbl_p, _c_dbl_p, ctypes.c_int64, ctypes.c_int64, _c_dbl_p, _c_dbl_p,
                                       _c_dbl_p]
        L.orc_rows_mult.restype = None
        L.orc_rows_mult.argtypes = [ctypes.c_int, _c_u32_p, ctypes.c_int64, _c_dbl_p, _c_dbl_p, ctypes.c_int,
                                    _c_int_p, _c_int_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, _c_dbl_p, ctypes.c_int64,
                                    ctypes.c_int64, _c_dbl_p, _c_dbl_p]
        L.orc_sample_times_mt.restype = None
        L.orc_sample_times_mt.argtypes = L.orc_sample_times.argtypes
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_num_threads.argtypes = []
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def basis(N: int, n_up: int) -> np.ndarray:
    """Sz-sector basis in the reference's order (odometer restatement)."""
    L = lib()
    D = L.orc_basis_build(N, n_up, None, 0)
    out = np.empty(D, dtype=np.uint32)
    L.orc_basis_build(N, n_up, _p(out, _c_u32_p), D)
    return out


def index(states: np.ndarray, s: int) -> int:
    states = np.ascontiguousarray(states, dtype=np.uint32)
    return lib().orc_index(_p(states, _c_u32_p), states.size, s)


def start_vector(seed: int, D: int) -> np.ndarray:
    out = np.empty(D, dtype=np.float64)
    lib().orc_start_vector(seed, D, _p(out, _c_dbl_p))
    return out


class Matrix:
    """Explicit sparse H built in the reference's element order (hamiltonian_matrix.hpp)."""

    def __init__(self, N, n_up, bonds, site_h=None, site_d=None):
        L = lib()
        nb = len(bonds)
        s1 = np.array([b[0] for b in bonds], dtype=np.int32)
        s2 = np.array([b[1] for b in bonds], dtype=np.int32)
        jz = np.array([b[2] for b in bonds], dtype=np.float64)
        jxy = np.array([b[3] for b in bonds], dtype=np.float64)
        kq = np.array([b[4] if len(b) > 4 else 0.0 for b in bonds], dtype=np.float64)
        sh = None if site_h is None else np.ascontiguousarray(site_h, dtype=np.float64)
        sd = None if site_d is None else np.ascontiguousarray(site_d, dtype=np.float64)
        self._h = L.orc_matrix_build(N, n_up, _p(sh, _c_dbl_p), _p(sd, _c_dbl_p), nb,
                                     _p(s1, _c_int_p), _p(s2, _c_int_p), _p(jz, _c_dbl_p),
                                     _p(jxy, _c_dbl_p), _p(kq, _c_dbl_p))
        if not self._h:
            raise ValueError("oracle: invalid model")
        self.N, self.n_up, self.bonds = N, n_up, bonds
        self.D = L.orc_matrix_dim(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_matrix_free(self._h)
            self._h = None

    @property
    def nnz(self):
        return lib().orc_matrix_nnz(self._h)

    def states(self):
        out = np.empty(self.D, dtype=np.uint32)
        lib().orc_matrix_states(self._h, _p(out, _c_u32_p))
        return out

    def csr(self):
        rp = np.empty(self.D + 1, dtype=np.int64)
        col = np.empty(self.nnz, dtype=np.int32)
        val = np.empty(self.nnz, dtype=np.float64)
        lib().orc_matrix_csr(self._h, _p(rp, _c_i64_p), _p(col, _c_i32_p), _p(val, _c_dbl_p))
        return rp, col, val

    def dense(self):
        rp, col, val = self.csr()
        M = np.zeros((self.D, self.D))
        for i in range(self.D):
            for p in range(rp[i], rp[i + 1]):
                M[i, col[p]] += val[p]
        return M

    def mult(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.D, dtype=np.float64)
        lib().orc_matrix_mult(self._h, _p(x, _c_dbl_p), _p(y, _c_dbl_p))
        return y

    def mult_rows(self, x, y, r0, r1):
        lib().orc_matrix_mult_rows(self._h, _p(x, _c_dbl_p), _p(y, _c_dbl_p), r0, r1)

    def lanczos(self, nev=1, max_iter=None, seed=0, start=None, rtol=None, atol=None, ab_cap=4096):
        """ietl::lanczos + lanczos_iteration_nlowest; returns dict."""
        eps = np.finfo(np.float64).eps
        rtol = 100 * eps if rtol is None else rtol
        atol = 100 * eps if atol is None else atol
        if max_iter is None:
            max_iter = min(10 * self.D, 1000)
        ev = np.zeros(max(nev, 1))
        er = np.zeros(max(nev, 1))
        it = ctypes.c_int(0)
        fail = ctypes.c_int(0)
        al = np.zeros(ab_cap)
        be = np.zeros(ab_cap)
        st = None if start is None else np.ascontiguousarray(start, dtype=np.float64)
        n = lib().orc_lanczos(self._h, nev, max_iter, seed, _p(st, _c_dbl_p), rtol, atol, _p(ev, _c_dbl_p),
                              _p(er, _c_dbl_p), ctypes.byref(it), ctypes.byref(fail), _p(al, _c_dbl_p),
                              _p(be, _c_dbl_p), ab_cap)
        if n < 0:
            raise RuntimeError(f"oracle lanczos failed ({n})")
        m = it.value
        return {"evals": ev[:n].copy(), "errors": er[:n].copy(), "iterations": m, "fail": fail.value,
                "alpha": al[:min(m, ab_cap)].copy(), "beta": be[:min(m, ab_cap)].copy()}


def stev(d, e, want_last=False, want_full=False):
    d = np.ascontiguousarray(d, dtype=np.float64)
    e = np.ascontiguousarray(e, dtype=np.float64)
    n = d.size
    w = np.empty(n)
    zl = np.empty(n) if want_last else None
    zf = np.empty(n * n) if want_full else None
    ee = np.zeros(max(n, 1))
    ee[: max(n - 1, 0)] = e[: max(n - 1, 0)]
    info = lib().orc_stev(n, _p(d, _c_dbl_p), _p(ee, _c_dbl_p), _p(w, _c_dbl_p), _p(zl, _c_dbl_p), _p(zf, _c_dbl_p))
    if info:
        raise RuntimeError("oracle stev failed")
    out = [w]
    if want_last:
        out.append(zl)
    if want_full:
        out.append(zf.reshape(n, n).T)  # columns = eigenvectors
    return out if len(out) > 1 else w


def tmatrix(alpha, beta, cap=4096):
    """Tmatrix::compute(true): distinct non-ghost eigenvalues, errors, multiplicities."""
    alpha = np.ascontiguousarray(alpha, dtype=np.float64)
    beta = np.ascontiguousarray(beta, dtype=np.float64)
    n = alpha.size
    ev = np.zeros(cap)
    er = np.zeros(cap)
    mu = np.zeros(cap, dtype=np.int32)
    th = ctypes.c_double(0)
    ml = ctypes.c_double(0)
    cnt = lib().orc_tmatrix(n, _p(alpha, _c_dbl_p), _p(beta, _c_dbl_p), _p(ev, _c_dbl_p), _p(er, _c_dbl_p),
                            _p(mu, _c_int_p), cap, ctypes.byref(th), ctypes.byref(ml))
    if cnt < 0:
        raise RuntimeError("oracle tmatrix failed")
    return {"evals": ev[:cnt].copy(), "errors": er[:cnt].copy(), "mults": mu[:cnt].copy(),
            "thold": th.value, "multol": ml.value}


def tmatrix_lapack(alpha, beta):
    """Tmatrix::compute(true) with LAPACK dstev itself (scipy), to pin tmatrix()."""
    from scipy.linalg import lapack

    alpha = np.asarray(alpha, dtype=np.float64)
    beta = np.asarray(beta, dtype=np.float64)
    n = alpha.size
    eps = np.finfo(np.float64).eps
    w, z, info = lapack.dstev(alpha.copy(), beta[: n - 1].copy(), compute_v=1)[:3]
    assert info == 0
    multol = max(alpha.max(), beta.max()) * 2 * eps * (10000 + n)
    thold = max(w[0], w[n - 1])
    thold = max(eps ** (2.0 / 3.0) * thold, 5 * multol)
    bl = beta[n - 1]
    distinct, mult, err = [w[0]], [], []
    temp, multiple = w[0], 1
    for i in range(1, n):
        if w[i] - temp > thold:
            distinct.append(w[i])
            temp = w[i]
            mult.append(multiple)
            err.append(0.0 if multiple > 1 else abs(bl * z[n - 1, i - 1]))
            multiple = 1
        else:
            multiple += 1
    mult.append(multiple)
    err.append(0.0 if multiple > 1 else abs(bl * z[n - 1, n - 1]))
    if n > 1:
        if n - 1 > 1:
            wg = lapack.dstev(alpha[1:].copy(), beta[1: n - 1].copy(), compute_v=0)[0]
        else:
            wg = alpha[1:].copy()
    else:
        wg = np.zeros(0)
    t2 = 0
    for i, k in enumerate(distinct):
        if mult[i] == 1:
            j = t2
            while j < n - 2:
                if wg[j] - k >= multol:
                    break
                if abs(k - wg[j]) < multol:
                    mult[i] = 0
                    err[i] = 0.0
                    t2 += 1
                    break
                j += 1
                t2 += 1
    keep = [i for i in range(len(distinct)) if mult[i] != 0]
    return {"evals": np.array([distinct[i] for i in keep]), "errors": np.array([err[i] for i in keep]),
            "mults": np.array([mult[i] for i in keep]), "thold": thold, "multol": multol}


def hv_matfree(N, states, bonds, x, r0=0, r1=None):
    """Matrix-free H*x with all host threads (best-CPU baseline), rows [r0, r1)."""
    states = np.ascontiguousarray(states, dtype=np.uint32)
    D = states.size
    r1 = D if r1 is None else r1
    s1 = np.array([b[0] for b in bonds], dtype=np.int32)
    s2 = np.array([b[1] for b in bonds], dtype=np.int32)
    jz = np.array([b[2] for b in bonds], dtype=np.float64)
    jxy = np.array([b[3] for b in bonds], dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(D)
    lib().orc_hv_matfree(N, _p(states, _c_u32_p), D, len(bonds), _p(s1, _c_int_p), _p(s2, _c_int_p),
                         _p(jz, _c_dbl_p), _p(jxy, _c_dbl_p), _p(x, _c_dbl_p), _p(y, _c_dbl_p), r0, r1)
    return y


def basis_fast(N: int, n_up: int) -> np.ndarray:
    """Same states as basis() (tested), enumerated by next-same-popcount stepping."""
    L = lib()
    D = L.orc_basis_fast(N, n_up, None, 0)
    out = np.empty(D, dtype=np.uint32)
    L.orc_basis_fast(N, n_up, _p(out, _c_u32_p), D)
    return out


def sample_times(N, states, bonds, r0, r1):
    """Seconds for the reference algorithm on rows [r0, r1): (matrix build, prod, vector passes)."""
    states = np.ascontiguousarray(states, dtype=np.uint32)
    s1 = np.array([b[0] for b in bonds], dtype=np.int32)
    s2 = np.array([b[1] for b in bonds], dtype=np.int32)
    jz = np.array([b[2] for b in bonds], dtype=np.float64)
    jxy = np.array([b[3] for b in bonds], dtype=np.float64)
    tb, tp, tv = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
    lib().orc_sample_times(N, _p(states, _c_u32_p), states.size, len(bonds), _p(s1, _c_int_p), _p(s2, _c_int_p),
                           _p(jz, _c_dbl_p), _p(jxy, _c_dbl_p), r0, r1, ctypes.byref(tb), ctypes.byref(tp),
                           ctypes.byref(tv))
    return tb.value, tp.value, tv.value


def sample_times_mt(N, states, bonds, r0, r1):
    """sample_times with all host threads (contiguous row blocks per thread): wall seconds of the
    matrix build, the row sums and the vector passes over rows [r0, r1)."""
    states = np.ascontiguousarray(states, dtype=np.uint32)
    s1 = np.array([b[0] for b in bonds], dtype=np.int32)
    s2 = np.array([b[1] for b in bonds], dtype=np.int32)
    jz = np.array([b[2] for b in bonds], dtype=np.float64)
    jxy = np.array([b[3] for b in bonds], dtype=np.float64)
    tb, tp, tv = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
    lib().orc_sample_times_mt(N, _p(states, _c_u32_p), states.size, len(bonds), _p(s1, _c_int_p), _p(s2, _c_int_p),
                              _p(jz, _c_dbl_p), _p(jxy, _c_dbl_p), r0, r1, ctypes.byref(tb), ctypes.byref(tp),
                              ctypes.byref(tv))
    return tb.value, tp.value, tv.value


def rows_mult(N, states, bonds, x, r0, r1, site_h=None, site_d=None):
    """Rows [r0, r1) of the explicit matrix (reference element order) times x, for sectors too large
    to build whole; ``states`` is the full sector (``basis_fast``), ``x`` the full vector.  Returns
    (y, sum_j |M_ij x_j|) over the window."""
    states = np.ascontiguousarray(states, dtype=np.uint32)
    D = states.size
    r1 = min(r1, D)
    s1 = np.array([b[0] for b in bonds], dtype=np.int32)
    s2 = np.array([b[1] for b in bonds], dtype=np.int32)
    jz = np.array([b[2] for b in bonds], dtype=np.float64)
    jxy = np.array([b[3] for b in bonds], dtype=np.float64)
    kq = np.array([b[4] if len(b) > 4 else 0.0 for b in bonds], dtype=np.float64)
    sh = None if site_h is None else np.ascontiguousarray(site_h, dtype=np.float64)
    sd = None if site_d is None else np.ascontiguousarray(site_d, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    assert x.size == D
    y = np.empty(r1 - r0)
    ya = np.empty(r1 - r0)
    lib().orc_rows_mult(N, _p(states, _c_u32_p), D, _p(sh, _c_dbl_p), _p(sd, _c_dbl_p), len(bonds),
                        _p(s1, _c_int_p), _p(s2, _c_int_p), _p(jz, _c_dbl_p), _p(jxy, _c_dbl_p),
                        _p(kq, _c_dbl_p), _p(x, _c_dbl_p), r0, r1, _p(y, _c_dbl_p), _p(ya, _c_dbl_p))
    return y, ya


def num_threads() -> int:
    return lib().orc_num_threads()
