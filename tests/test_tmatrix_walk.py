"""Host checks of the T-matrix algorithms the batched engine runs on the GPU (no GPU needed).

The batched check finds the low end of T's spectrum by Sturm-count bisection (a lane per
eigenvalue), walks Tmatrix::compute's distinct / ghost rules over the prefixes it has
(tcore::walk_prefix, growing them when the walk needs more) and takes the error estimates'
eigenvector components from inverse iteration; the single-instance path uses the QL sweeps of
tcore::analyze.  A small C++ driver compiled from the engine's own header runs both on Lanczos
T-matrices with ghost copies (FP32 and FP64 recurrences of an L=14 chain, from the oracle's
explicit matrix): the same distinct values, multiplicities and first indices, values within a
few ulps of |T|, error estimates within 1e-3.  The Rayleigh-Ritz pencil routine (rr_core.h) is
checked against LAPACK on random pencils, including a nearly dependent pair of vectors.
"""

import os
import subprocess
import tempfile

import numpy as np
import scipy.linalg

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "alps_b200", "csrc")

WALK_DRIVER = r"""
#include <algorithm>
#include <cstdio>
#include <vector>
#include "tmatrix_core.h"
using namespace aed;
int main(int argc, char** argv) {
  int m, nev, tr;
  std::vector<double> A, B;
  while (std::scanf("%d %d %d", &m, &nev, &tr) == 3) {
    A.assign(m, 0.0); B.assign(m, 0.0);
    for (int i = 0; i < m; ++i) std::scanf("%lf %lf", &A[i], &B[i]);
    const double thold_rel = tr ? 2e-6 : 0.0;
    const int want = nev + 1;
    double amax = A[0], bmax = B[0];
    for (int q = 0; q < m; ++q) { amax = std::max(amax, A[q]); bmax = std::max(bmax, B[q]); }
    std::vector<double> scratch(5 * m + 32);
    double ev[40], er[40]; int mu[40], fi[40]; tcore::TResult res;
    tcore::analyze(m, A.data(), B.data(), amax, bmax, scratch.data(), want, ev, er, mu, fi, &res, thold_rel);
    double glo, ghi, g2l, g2h;
    tcore::gershgorin(A.data(), B.data(), m, &glo, &ghi);
    tcore::gershgorin(A.data() + 1, B.data() + 1, m - 1, &g2l, &g2h);
    const double top = tcore::bisect_eigenvalue(A.data(), B.data(), m, m - 1, glo, ghi);
    std::vector<double> evt(m), evg(m);
    int nt = std::min(m, want + 4), ng = std::min(m - 1, want + 5), pt = 0, pg = 0, n = -1;
    tcore::WalkItem it[40]; double th, mt;
    for (int round = 0; round < 4 && n < 0; ++round) {
      for (int k = pt; k < nt; ++k) evt[k] = tcore::bisect_eigenvalue(A.data(), B.data(), m, k, glo, ghi);
      for (int k = pg; k < ng; ++k) evg[k] = tcore::bisect_eigenvalue(A.data() + 1, B.data() + 1, m - 1, k, g2l, g2h);
      n = tcore::walk_prefix(m, amax, bmax, evt.data(), nt, top, evg.data(), ng, want, thold_rel, it, &th, &mt);
      pt = nt; pg = ng;
      nt = std::min(m, 2 * nt + 4); ng = std::min(m - 1, 2 * ng + 4);
    }
    std::printf("%d %d", res.count, n);
    for (int q = 0; q < res.count; ++q) std::printf(" %.17g %.17g %d %d", ev[q], er[q], mu[q], fi[q]);
    for (int q = 0; q < (n > 0 ? n : 0); ++q) {
      double e2 = 0.0;
      if (it[q].zidx >= 0) {
        std::vector<double> z(m), sc(6 * m);
        tcore::inverse_iteration(m, A.data(), B.data(), evt[it[q].zidx], z.data(), sc.data());
        e2 = std::fabs(B[m - 1] * z[m - 1]);
      }
      std::printf(" %.17g %.17g %d %d", it[q].value, e2, it[q].mult, it[q].first);
    }
    std::printf(" %.17g\n", std::max(std::fabs(glo), std::fabs(ghi)));
  }
}
"""

RR_DRIVER = r"""
#include <cstdio>
#include "rr_core.h"
using namespace aed;
int main() {
  int K;
  while (std::scanf("%d", &K) == 1) {
    double G[64], A[64];
    for (int i = 0; i < K * K; ++i) std::scanf("%lf", &G[i]);
    for (int i = 0; i < K * K; ++i) std::scanf("%lf", &A[i]);
    double th[8], cr[8][8]; int ord[8];
    const int Kp = rrcore::ritz_pairs(K, G, A, th, cr, ord);
    std::printf("%d", Kp);
    for (int i = 0; i < Kp; ++i) std::printf(" %.17g", th[ord[i]]);
    std::printf("\n");
  }
}
"""


def _build(src, name, tmp):
    path = os.path.join(tmp, name + ".cpp")
    with open(path, "w") as f:
        f.write(src)
    exe = os.path.join(tmp, name)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, path, "-o", exe], check=True, capture_output=True)
    return exe


def _lanczos_tmatrices():
    """alpha, beta of plain Lanczos (no reorthogonalisation) on an L=14 chain in FP32 and FP64 vectors:
    the FP32 runs hold ghost copies of the converged values."""
    L = 14
    M = oracle.Matrix(L, L // 2, [(i, (i + 1) % L, 1.0, 1.0, 0.0) for i in range(L)])
    rng = np.random.default_rng(5)
    out = []
    for steps, dt in [(140, np.float32), (100, np.float32), (60, np.float64)]:
        v = rng.normal(size=M.D).astype(dt)
        v /= np.linalg.norm(v)
        vp = np.zeros_like(v)
        beta = 0.0
        A, B = [], []
        for _ in range(steps):
            w = M.mult(v.astype(np.float64)).astype(dt)
            a = float(np.dot(v.astype(np.float64), w.astype(np.float64)))
            w = (w - a * v - beta * vp).astype(dt)
            beta = float(np.linalg.norm(w.astype(np.float64)))
            A.append(a)
            B.append(beta)
            vp, v = v, (w / beta).astype(dt)
        out.append((np.array(A), np.array(B)))
    return out


def test_bisection_walk_matches_the_ql_analysis():
    cases = []
    for A, B in _lanczos_tmatrices():
        for m in range(4, len(A) + 1, 4):
            for nev in (1, 2, 4):
                for tr in (0, 1):
                    cases.append((m, nev, tr, A[:m], B[:m]))
    text = "".join(f"{m} {nev} {tr}\n" + "".join(f"{a:.17g} {b:.17g}\n" for a, b in zip(A, B)) for m, nev, tr, A, B in cases)
    with tempfile.TemporaryDirectory() as tmp:
        exe = _build(WALK_DRIVER, "walk", tmp)
        out = subprocess.run([exe], input=text, capture_output=True, text=True, check=True).stdout.splitlines()
    assert len(out) == len(cases)
    for line, (m, nev, tr, _, _) in zip(out, cases):
        f = line.split()
        nq, nb = int(f[0]), int(f[1])
        assert nb == nq, (m, nev, tr, line[:200])  # the prefixes sufficed, and the same number of values
        ref = [f[2 + 4 * q: 6 + 4 * q] for q in range(nq)]
        got = [f[2 + 4 * nq + 4 * q: 6 + 4 * nq + 4 * q] for q in range(nb)]
        scale = float(f[-1])
        for (v0, e0, m0, f0), (v1, e1, m1, f1) in zip(ref, got):
            assert (m0, f0) == (m1, f1), (m, nev, tr)
            assert abs(float(v0) - float(v1)) <= 64 * np.finfo(float).eps * scale, (m, nev, tr, v0, v1)
            e0, e1 = float(e0), float(e1)
            assert abs(e0 - e1) <= 1e-3 * max(e0, 1e-12 * scale), (m, nev, tr, e0, e1)


def test_ritz_pairs_match_lapack_on_random_pencils():
    rng = np.random.default_rng(9)
    cases = []
    for K in (1, 2, 3, 5, 8):
        X = rng.normal(size=(40, K))
        H = rng.normal(size=(40, 40))
        H = H + H.T
        cases.append((K, X.T @ X, X.T @ H @ X, None))
    # a nearly dependent pair (a vector and its slightly perturbed copy): one direction is dropped or
    # gives a value far from the pencil's others; the well-conditioned values are kept
    X = rng.normal(size=(40, 3))
    X[:, 2] = X[:, 1] + 1e-7 * rng.normal(size=40)
    H = np.diag(np.arange(40.0))
    cases.append((3, X.T @ X, X.T @ H @ X, X[:, :2]))
    text = "".join(f"{K}\n" + " ".join(f"{v:.17g}" for v in G.ravel()) + "\n" + " ".join(f"{v:.17g}" for v in A.ravel()) + "\n"
                   for K, G, A, _ in cases)
    with tempfile.TemporaryDirectory() as tmp:
        exe = _build(RR_DRIVER, "rr", tmp)
        out = subprocess.run([exe], input=text, capture_output=True, text=True, check=True).stdout.splitlines()
    for line, (K, G, A, base) in zip(out, cases):
        f = line.split()
        Kp, th = int(f[0]), np.array([float(v) for v in f[1:]])
        if base is None:
            assert Kp == K
            ref = scipy.linalg.eigh(A, G, eigvals_only=True)
            np.testing.assert_allclose(th, ref, rtol=1e-9, atol=1e-9 * np.max(np.abs(ref)))
        else:
            # the span of the two independent vectors: its Ritz values must be among the results
            Gb, Ab = base.T @ base, base.T @ H @ base
            ref = scipy.linalg.eigh(Ab, Gb, eigvals_only=True)
            for r in ref:
                assert np.min(np.abs(th - r)) <= 1e-6 * max(abs(r), 1.0), (th, ref)
