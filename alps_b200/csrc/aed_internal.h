// aed_internal.h -- shared declarations of the engine's host and device code.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/aed.h"

namespace aed {

// ---- errors ----------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

#define AED_CUDA_TRY(expr)                                                                  \
  do {                                                                                      \
    cudaError_t aed_e_ = (expr);                                                            \
    if (aed_e_ != cudaSuccess)                                                              \
      return ::aed::fail(AED_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(aed_e_)); \
  } while (0)

constexpr int kMaxBonds = AED_MAX_BONDS;
constexpr int kMaxDiag = AED_MAX_BONDS + 32;

// ---- host model ------------------------------------------------------------
struct Model {
  int N = 0, n_up = 0;
  std::vector<int> s1, s2;
  std::vector<double> jz, jxy, kq;
  std::vector<double> site_h, site_d;  // empty when absent
};

int model_from_desc(const aed_model_desc* d, Model& m);

// ---- device-facing coupling tables -------------------------------------------
// A spin-flip pair: bits mhi > mlo (masks), merged coefficient of all bonds
// joining the two sites, summed in bond order.
struct PairTerm {
  uint32_t mhi, mlo;
  double c;
  float chi, clo;  // c split into two floats (c ~= chi + clo) for the FP32 kernels
};

// One diagonal contribution, in the reference's accumulation order (site
// terms, then bonds): v = ((s & m1) != 0) == ((s & m2) != 0) ? veq : vne.
// A site term uses m2 = 0, so veq is its Sz = -1/2 value and vne its +1/2 value.
struct DiagTerm {
  uint32_t m1, m2;
  double veq, vne;
};

struct HvParams {
  int N, Nlo, n_up;
  int n_pairs;  // entries in low[] and rise[]
  int n_diag;
  uint32_t lomask;
  // pairs in ascending-column order for a row: "low" flips (target < source)
  // sorted by (hi desc, lo asc); "rise" flips (target > source) by (hi asc, lo desc)
  PairTerm low[kMaxBonds];
  PairTerm rise[kMaxBonds];
  DiagTerm diag[kMaxDiag];
  // flips with both bits in the lo part, in the order of low[]: their
  // coefficients, indexed by the lo-neighbour table
  int n_lolo;
  double lolo_c[kMaxBonds];
};

int build_hv_params(const Model& m, int Nlo, HvParams& P);

// ---- basis tables ----------------------------------------------------------
// Lin two-table ranking: rank(s) = thi[s >> Nlo] + tlo[s & lomask].
struct BasisTables {
  int N = 0, n_up = 0, Nlo = 0, Nhi = 0;
  int64_t D = 0;
  std::vector<uint32_t> thi;     // 2^Nhi: states before hi block h
  std::vector<uint16_t> tlo;     // 2^Nlo: rank of l among same-popcount lo values
  std::vector<uint16_t> lolist;  // 2^Nlo: lo values grouped by popcount, ascending
  std::vector<uint32_t> looff;   // Nlo+2 offsets into lolist per popcount
};

int build_tables(int N, int n_up, BasisTables& t);

// Lo-neighbour table: for every lo state l (rank r within its popcount class
// k), the flips with both bits in the lo part that apply to l, as
// (target rank r' = tlo[l ^ flip]) | (flip index << 16), sorted by r' and
// padded with kEllPad to a common width W.  Entry e of row r of class k sits
// at W * looff[k] + e * C(Nlo, k) + r (coalesced across consecutive rows).
constexpr uint32_t kEllPad = 0xffffffffu;
void build_lo_table(const BasisTables& t, const HvParams& P, std::vector<uint32_t>& ell, int* width);

// Work tiles over the sector: (hi block h, first row r0 within the block).
void build_tiles(const BasisTables& t, int tile_rows, std::vector<uint32_t>& th, std::vector<uint32_t>& tr,
                 std::vector<uint32_t>* tfirst = nullptr);
// Hi blocks grouped by lo popcount (largest blocks first, bit-reversed h
// ascending within a group), each group padded with kNoBlockEntry to a multiple of kBundleMax, so
// that bundles of 1, 2 or 4 consecutive entries never mix groups.  *maxrows:
// rows of the largest block.
// Crossing-flip table: entry b * 2^Nlo + looff[k] + r is the rank (within
// its popcount class) of lo state lolist[looff[k] + r] with bit b flipped,
// with bit 15 = the state's bit b (ranks are below 2^15 for Nlo <= 16).
void build_cross_table(const BasisTables& t, std::vector<uint16_t>& xt);
constexpr int kBundleMax = 4;
constexpr uint32_t kNoBlockEntry = 0xffffffffu;
void build_block_list(const BasisTables& t, std::vector<uint32_t>& blk, int* maxrows);

// ---- tridiagonal / Tmatrix (host) ---------------------------------------------
int tridiag_eigen(int n, double* d, double* e, double* zlast, double* zfull = nullptr);

struct TmatInfo {
  std::vector<double> evals, errs;  // distinct, non-ghost
  std::vector<int> mults;
  std::vector<int> first;           // index of each value in the sorted T spectrum
  double thold = 0, multol = 0;
};
int tmatrix_analyze(int n, const double* alpha, const double* beta, double alpha_max, double beta_max,
                    TmatInfo& out, double thold_rel = 0.0);
// merge threshold (relative) of T-matrix analyses of FP32 recurrences
constexpr double kFp32MergeRel = 2e-6;
bool nlowest_converged(const TmatInfo& t, int nev, double rtol, double atol);

// ---- parameters / lattices ----------------------------------------------------
struct ParsedParams {
  aed_param_info info;
  std::vector<int> s1, s2;
  std::vector<double> jz, jxy, kq, site_h, site_d;
};
// A graph of a lattice library (<GRAPH>, src/alps/lattice/graph.h:121-222):
// n vertices with their types, edges (source, target, type) in file order,
// vertices numbered from 0.
struct GraphSpec {
  int n = 0;
  std::vector<int> vtype, src, tgt, etype;
};
// graph == nullptr: the lattice the parameters name.
int parse_parameters(const char* text, ParsedParams& out, const GraphSpec* graph = nullptr);
// Lattice dimension, extents and periodic flags of the parameters.
int lattice_geometry(const char* text, int* dim, int ext[2], int periodic[2]);
// Momenta the sector loop visits (diag.h:93-114): TOTAL_MOMENTUM when given,
// else every translation momentum when TRANSLATION_SYMMETRY (default true),
// else none.  *n_dirs = periodic directions of the lattice.
int lattice_momenta(const char* text, int* n_dirs, std::vector<std::vector<double>>& ks);
// Translations of the lattice at momentum k: maps (n_trans x n_sites, site i
// goes to maps[t * n_sites + i]) and phases exp(i k.R_t).
int lattice_translations(const char* text, const double* k, int n_k, int* n_sites, std::vector<int>& maps,
                         std::vector<double>& re, std::vector<double>& im);

}  // namespace aed
