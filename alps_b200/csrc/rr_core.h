// rr_core.h -- the small dense part of the Rayleigh-Ritz refinement, for the
// host (single-instance solves) and the device (the batched engine, one
// thread per request).
//
// Given K FP64 vectors Psi (the Ritz vectors of the FP32 phase's T that span
// its nev lowest clusters) with Gram matrix G = Psi^T Psi and projection
// A = Psi^T H Psi, the Ritz pairs of H on span(Psi): G's nearly dependent
// directions are dropped (a ghost copy of a converged vector leaves one),
// the projected problem is solved in the orthonormalised basis by cyclic
// Jacobi, and each value is taken as the Rayleigh quotient c^T A c / c^T G c
// of its own coefficients c (so the conditioning of the basis cannot move
// it).  The caller then forms the residuals |H Psi c - theta Psi c| of the
// pairs below the gap bound on the device and applies the block Kato-Temple
// bound.  Plain pointers and fixed-size arrays; no allocation.
#pragma once

#include <cmath>

#ifndef AED_HD
#ifdef __CUDACC__
#define AED_HD __host__ __device__
#else
#define AED_HD
#endif
#endif

namespace aed {
namespace rrcore {

constexpr int kMax = 8;  // Ritz vectors in one refinement (kMaxRR)

// Eigen-decomposition of a symmetric n x n matrix a (row-major, destroyed) by
// cyclic Jacobi rotations (Jacobi 1846; the threshold-free cyclic form of
// Rutishauser, Handbook for Automatic Computation II, 1971): w ascending,
// column k of v (v[i * n + k]) its eigenvector.  n <= kMax.
AED_HD inline void jacobi_eigen(int n, double* a, double* w, double* v) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) v[i * n + j] = i == j ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int i = 0; i < n; ++i) {
      diag += a[i * n + i] * a[i * n + i];
      for (int j = i + 1; j < n; ++j) off += a[i * n + j] * a[i * n + j];
    }
    if (off <= 1e-34 * diag || off == 0.0) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[p * n + q];
        if (apq == 0.0) continue;
        // rotation angle that zeroes a_pq: tan(phi) = t, the smaller root of t^2 + 2 theta t - 1 = 0
        const double theta = (a[q * n + q] - a[p * n + p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {  // columns p, q
          const double akp = a[k * n + p], akq = a[k * n + q];
          a[k * n + p] = c * akp - s * akq;
          a[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // rows p, q
          const double apk = a[p * n + k], aqk = a[q * n + k];
          a[p * n + k] = c * apk - s * aqk;
          a[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = v[k * n + p], vkq = v[k * n + q];
          v[k * n + p] = c * vkp - s * vkq;
          v[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  // ascending order (stable selection of the diagonal)
  int ord[kMax];
  for (int i = 0; i < n; ++i) ord[i] = i;
  for (int i = 1; i < n; ++i) {
    const int o = ord[i];
    int j = i - 1;
    while (j >= 0 && a[ord[j] * n + ord[j]] > a[o * n + o]) {
      ord[j + 1] = ord[j];
      --j;
    }
    ord[j + 1] = o;
  }
  double vs[kMax * kMax];
  for (int k = 0; k < n; ++k) {
    w[k] = a[ord[k] * n + ord[k]];
    for (int i = 0; i < n; ++i) vs[i * n + k] = v[i * n + ord[k]];
  }
  for (int i = 0; i < n * n; ++i) v[i] = vs[i];
}

// x^T M y for K x K row-major M.
AED_HD inline double form(int K, const double* M, const double* x, const double* y) {
  double s = 0.0;
  for (int a = 0; a < K; ++a)
    for (int b = 0; b < K; ++b) s += x[a] * M[a * K + b] * y[b];
  return s;
}

// Ritz pairs of the pencil (A, G), K x K row-major (A symmetrised here).
// th[q], cr[q][0..K): value and coefficients over Psi of pair q; ord: the
// pairs by ascending value.  Returns the number of pairs Kp (0: G is not
// positive).
AED_HD inline int ritz_pairs(int K, const double* G, const double* A_in, double* th, double (*cr)[kMax], int* ord) {
  double A[kMax * kMax], Gc[kMax * kMax], g[kMax], Q[kMax * kMax];
  for (int i = 0; i < K * K; ++i) {
    A[i] = A_in[i];
    Gc[i] = G[i];
  }
  for (int a = 0; a < K; ++a)
    for (int b = a + 1; b < K; ++b) A[a * K + b] = A[b * K + a] = 0.5 * (A[a * K + b] + A[b * K + a]);
  jacobi_eigen(K, Gc, g, Q);
  const double gmax = g[K - 1];
  if (!(gmax > 0)) return 0;
  // orthonormal basis of span(Psi): B = Q_kept diag(g)^{-1/2}
  double B[kMax * kMax];
  int Kp = 0;
  for (int k = K - 1; k >= 0; --k) {
    if (!(g[k] > 1e-10 * gmax)) continue;
    const double s = 1.0 / sqrt(g[k]);
    for (int i = 0; i < K; ++i) B[i * K + Kp] = Q[i * K + k] * s;
    ++Kp;
  }
  // C = B^T A B (Kp x Kp)
  double AB[kMax * kMax], C[kMax * kMax], Y[kMax * kMax];
  for (int i = 0; i < K; ++i)
    for (int j = 0; j < Kp; ++j) {
      double s = 0.0;
      for (int k = 0; k < K; ++k) s += A[i * K + k] * B[k * K + j];
      AB[i * K + j] = s;
    }
  for (int i = 0; i < Kp; ++i)
    for (int j = 0; j < Kp; ++j) {
      double s = 0.0;
      for (int k = 0; k < K; ++k) s += B[k * K + i] * AB[k * K + j];
      C[i * Kp + j] = s;
    }
  for (int i = 0; i < Kp; ++i)
    for (int j = i + 1; j < Kp; ++j) C[i * Kp + j] = C[j * Kp + i] = 0.5 * (C[i * Kp + j] + C[j * Kp + i]);
  jacobi_eigen(Kp, C, th, Y);
  for (int q = 0; q < Kp; ++q) {
    for (int k = 0; k < K; ++k) {
      double s = 0.0;
      for (int j = 0; j < Kp; ++j) s += B[k * K + j] * Y[j * Kp + q];
      cr[q][k] = s;
    }
    const double den = form(K, G, cr[q], cr[q]);
    if (den > 0) th[q] = form(K, A, cr[q], cr[q]) / den;
    ord[q] = q;
  }
  for (int i = 1; i < Kp; ++i) {  // by value, stable
    const int o = ord[i];
    int j = i - 1;
    while (j >= 0 && th[ord[j]] > th[o]) {
      ord[j + 1] = ord[j];
      --j;
    }
    ord[j + 1] = o;
  }
  return Kp;
}

}  // namespace rrcore
}  // namespace aed
