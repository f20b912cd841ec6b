// model.cpp -- model description, coupling tables, basis tables, parameter surface.
//
// Reference paths are relative to the ALPS source tree.

#include <algorithm>
#include <cctype>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <sstream>
#include <stdexcept>

#include "aed_internal.h"

namespace aed {

// ---- errors ------------------------------------------------------------------
static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

const char* last_error_cstr() { return g_last_error.c_str(); }

// ---- model ---------------------------------------------------------------------
int model_from_desc(const aed_model_desc* d, Model& m) {
  if (!d) return fail(AED_ERR_INVALID, "model is NULL");
  if (d->n_sites < 2 || d->n_sites > 32) return fail(AED_ERR_INVALID, "n_sites must be in 2..32");
  if (d->n_up < 0 || d->n_up > d->n_sites) return fail(AED_ERR_INVALID, "n_up out of range");
  if (d->n_bonds < 0 || d->n_bonds > kMaxBonds) return fail(AED_ERR_INVALID, "n_bonds must be in 0..128");
  if (d->n_bonds > 0 && (!d->bond_s1 || !d->bond_s2 || !d->bond_jz || !d->bond_jxy))
    return fail(AED_ERR_INVALID, "bond arrays are NULL");
  m = Model();
  m.N = d->n_sites;
  m.n_up = d->n_up;
  for (int b = 0; b < d->n_bonds; ++b) {
    const int a = d->bond_s1[b], c = d->bond_s2[b];
    if (a < 0 || a >= m.N || c < 0 || c >= m.N || a == c)
      return fail(AED_ERR_INVALID, "bond " + std::to_string(b) + " has invalid sites");
    const double jz = d->bond_jz[b], jxy = d->bond_jxy[b], k = d->bond_k ? d->bond_k[b] : 0.0;
    if (!std::isfinite(jz) || !std::isfinite(jxy) || !std::isfinite(k))
      return fail(AED_ERR_INVALID, "bond " + std::to_string(b) + " has a non-finite coupling");
    m.s1.push_back(a);
    m.s2.push_back(c);
    m.jz.push_back(jz);
    m.jxy.push_back(jxy);
    m.kq.push_back(k);
  }
  if (d->site_h || d->site_d) {
    m.site_h.assign(m.N, 0.0);
    m.site_d.assign(m.N, 0.0);
    for (int s = 0; s < m.N; ++s) {
      if (d->site_h) m.site_h[s] = d->site_h[s];
      if (d->site_d) m.site_d[s] = d->site_d[s];
      if (!std::isfinite(m.site_h[s]) || !std::isfinite(m.site_d[s]))
        return fail(AED_ERR_INVALID, "non-finite site term");
    }
  }
  return AED_OK;
}

// Matrix elements of the spin-1/2 "spin" HAMILTONIAN (lib/xml/models.xml.in:342-373)
// as the reference's model library evaluates them (test/model/example3.output):
// site  Sz=-1/2: 0.25*D + 0.5*h;   Sz=+1/2: 0.25*D - 0.5*h
// bond  parallel: 0.25*Jz + 0.0625*K;  antiparallel: -0.25*Jz + 0.3125*K;
//       flip: 0.5*Jxy - 0.25*K
int build_hv_params(const Model& m, int Nlo, HvParams& P) {
  std::memset(&P, 0, sizeof P);
  P.N = m.N;
  P.Nlo = Nlo;
  P.n_up = m.n_up;
  P.lomask = (Nlo >= 32) ? 0xffffffffu : ((1u << Nlo) - 1u);
  const int nb = (int)m.s1.size();
  // diagonal terms in the reference's order: sites, then bonds
  // (hamiltonian_matrix.hpp:387-397); zero elements are skipped by
  // numeric::is_nonzero (hamiltonian_matrix.hpp:277,317) and adding +0.0 to
  // the accumulator is exact, so zero terms are simply dropped.
  int nd = 0;
  if (!m.site_h.empty()) {
    for (int s = 0; s < m.N; ++s) {
      const double vdown = 0.25 * m.site_d[s] + 0.5 * m.site_h[s];
      const double vup = 0.25 * m.site_d[s] - 0.5 * m.site_h[s];
      if (vdown == 0.0 && vup == 0.0) continue;
      if (nd >= kMaxDiag) return fail(AED_ERR_INVALID, "too many diagonal terms");
      P.diag[nd++] = {1u << (m.N - 1 - s), 0u, vdown, vup};
    }
  }
  for (int b = 0; b < nb; ++b) {
    const double par = 0.25 * m.jz[b] + 0.0625 * m.kq[b];
    const double anti = -0.25 * m.jz[b] + 0.3125 * m.kq[b];
    if (par == 0.0 && anti == 0.0) continue;
    if (nd >= kMaxDiag) return fail(AED_ERR_INVALID, "too many diagonal terms");
    P.diag[nd++] = {1u << (m.N - 1 - m.s1[b]), 1u << (m.N - 1 - m.s2[b]), par, anti};
  }
  P.n_diag = nd;
  // flip pairs, merged over bonds joining the same two sites in bond order
  // (matrix_as_vector.hpp:72-73 accumulates M(i,j) += v starting from 0)
  std::vector<PairTerm> pairs;
  for (int b = 0; b < nb; ++b) {
    const double flip = 0.5 * m.jxy[b] - 0.25 * m.kq[b];
    if (flip == 0.0) continue;
    uint32_t ma = 1u << (m.N - 1 - m.s1[b]), mb = 1u << (m.N - 1 - m.s2[b]);
    const uint32_t mhi = std::max(ma, mb), mlo = std::min(ma, mb);
    bool merged = false;
    for (auto& p : pairs)
      if (p.mhi == mhi && p.mlo == mlo) {
        p.c += flip;
        merged = true;
        break;
      }
    if (!merged) pairs.push_back({mhi, mlo, 0.0 + flip, 0.f, 0.f});
  }
  for (auto& p : pairs) {
    p.chi = (float)p.c;
    p.clo = (float)(p.c - (double)p.chi);
  }
  P.n_pairs = (int)pairs.size();
  std::vector<PairTerm> low = pairs, rise = pairs;
  // target < source (hi bit 1 -> 0): s' = s - 2^hi + 2^lo, ascending in
  // s' means hi descending, then lo ascending
  std::sort(low.begin(), low.end(), [](const PairTerm& a, const PairTerm& b) {
    return a.mhi != b.mhi ? a.mhi > b.mhi : a.mlo < b.mlo;
  });
  // target > source: s' = s + 2^hi - 2^lo, ascending means hi ascending, then lo descending
  std::sort(rise.begin(), rise.end(), [](const PairTerm& a, const PairTerm& b) {
    return a.mhi != b.mhi ? a.mhi < b.mhi : a.mlo > b.mlo;
  });
  for (int i = 0; i < P.n_pairs; ++i) {
    P.low[i] = low[i];
    P.rise[i] = rise[i];
  }
  P.n_lolo = 0;
  for (int i = 0; i < P.n_pairs; ++i)
    if ((P.low[i].mhi >> Nlo) == 0u) P.lolo_c[P.n_lolo++] = P.low[i].c;
  return AED_OK;
}

void build_lo_table(const BasisTables& t, const HvParams& P, std::vector<uint32_t>& ell, int* width) {
  std::vector<uint32_t> flips;
  for (int i = 0; i < P.n_pairs; ++i)
    if ((P.low[i].mhi >> t.Nlo) == 0u) flips.push_back(P.low[i].mhi | P.low[i].mlo);
  const uint32_t nlo = 1u << t.Nlo;
  // width: most flips applying to one lo state
  int W = 0;
  for (uint32_t l = 0; l < nlo; ++l) {
    int c = 0;
    for (uint32_t f : flips) {
      const uint32_t b = l & f;
      c += (b != 0u && b != f) ? 1 : 0;
    }
    W = std::max(W, c);
  }
  *width = W;
  ell.assign((size_t)W * nlo, kEllPad);
  std::vector<std::pair<uint32_t, uint32_t>> row;
  for (int k = 0; k <= t.Nlo; ++k) {
    const uint32_t base = t.looff[k], nk = t.looff[k + 1] - t.looff[k];
    for (uint32_t r = 0; r < nk; ++r) {
      const uint32_t l = t.lolist[base + r];
      row.clear();
      for (uint32_t q = 0; q < flips.size(); ++q) {
        const uint32_t b = l & flips[q];
        if (b != 0u && b != flips[q]) row.push_back({(uint32_t)t.tlo[l ^ flips[q]], q});
      }
      std::sort(row.begin(), row.end());
      for (size_t e = 0; e < row.size(); ++e)
        ell[(size_t)W * base + e * nk + r] = row[e].first | (row[e].second << 16);
    }
  }
}

void build_cross_table(const BasisTables& t, std::vector<uint16_t>& xt) {
  const uint32_t nlo = 1u << t.Nlo;
  xt.assign((size_t)t.Nlo * nlo, 0);
  for (int b = 0; b < t.Nlo; ++b)
    for (uint32_t i = 0; i < nlo; ++i) {
      const uint32_t l = t.lolist[i];
      xt[(size_t)b * nlo + i] = (uint16_t)(t.tlo[l ^ (1u << b)] | (((l >> b) & 1u) << 15));
    }
}

// ---- basis tables (Lin 1990 two-table ranking) -----------------------------------
static inline int popc32(uint32_t v) { return __builtin_popcount(v); }

int build_tables(int N, int n_up, BasisTables& t) {
  if (N < 2 || N > 32 || n_up < 0 || n_up > N) return fail(AED_ERR_INVALID, "bad sector");
  t = BasisTables();
  t.N = N;
  t.n_up = n_up;
  // lo part: half the sites, but at least 12 (two below N): hi blocks of a few
  // hundred to a thousand rows, the lo-part flips read from shared memory.
  // Small sectors with few rows per block paid a per-block overhead (program
  // compile, staging, barriers) on few rows: 12 made the 512-chain batch
  // 20-32 % faster than ceil(N/2) (11: 5-12 %, 13: FP64 only) and the
  // single-instance apply of L = 18-22 up to 25 % faster.
  t.Nlo = std::max((N + 1) / 2, std::min(12, N - 2));
  t.Nhi = N - t.Nlo;
  if (t.Nlo > 16) return fail(AED_ERR_INVALID, "N too large for 16-bit lo tables");
  const uint32_t nlo = 1u << t.Nlo, nhi = 1u << t.Nhi;
  std::vector<uint32_t> cnt(t.Nlo + 2, 0);
  for (uint32_t l = 0; l < nlo; ++l) cnt[popc32(l)]++;
  t.looff.assign(t.Nlo + 2, 0);
  for (int k = 0; k <= t.Nlo; ++k) t.looff[k + 1] = t.looff[k] + cnt[k];
  t.tlo.assign(nlo, 0);
  t.lolist.assign(nlo, 0);
  std::vector<uint32_t> fill(t.Nlo + 1, 0);
  for (uint32_t l = 0; l < nlo; ++l) {
    const int k = popc32(l);
    t.tlo[l] = (uint16_t)fill[k];
    t.lolist[t.looff[k] + fill[k]] = (uint16_t)l;
    fill[k]++;
  }
  t.thi.assign(nhi, 0);
  int64_t acc = 0;
  for (uint32_t h = 0; h < nhi; ++h) {
    t.thi[h] = (uint32_t)acc;
    const int k = n_up - popc32(h);
    if (k >= 0 && k <= t.Nlo) acc += cnt[k];
  }
  t.D = acc;
  if (acc > 0xffffffffll) return fail(AED_ERR_INVALID, "sector too large");
  return AED_OK;
}

void build_tiles(const BasisTables& t, int tile_rows, std::vector<uint32_t>& th, std::vector<uint32_t>& tr,
                 std::vector<uint32_t>* tfirst) {
  th.clear();
  tr.clear();
  const uint32_t nhi = 1u << t.Nhi;
  if (tfirst) tfirst->assign(nhi, 0u);
  for (uint32_t h = 0; h < nhi; ++h) {
    const int k = t.n_up - popc32(h);
    if (k < 0 || k > t.Nlo) continue;
    if (tfirst) (*tfirst)[h] = (uint32_t)th.size();
    const uint32_t rows = t.looff[k + 1] - t.looff[k];
    for (uint32_t r = 0; r < rows; r += tile_rows) {
      th.push_back(h);
      tr.push_back(r);
    }
  }
}

void build_block_list(const BasisTables& t, std::vector<uint32_t>& blk, int* maxrows) {
  blk.clear();
  *maxrows = 0;
  const uint32_t nhi = 1u << t.Nhi;
  std::vector<int> ks;
  for (int k = 0; k <= t.Nlo; ++k) {
    const int hk = t.n_up - k;  // popcount of the hi blocks with lo popcount k
    if (hk < 0 || hk > t.Nhi) continue;
    ks.push_back(k);
    *maxrows = std::max(*maxrows, (int)(t.looff[k + 1] - t.looff[k]));
  }
  std::stable_sort(ks.begin(), ks.end(), [&](int a, int b) {
    return t.looff[a + 1] - t.looff[a] > t.looff[b + 1] - t.looff[b];
  });
  // within a class, blocks in the order of their bit-reversed hi part: the
  // low hi bits change slowest, so flips of the top hi bits (the first sites)
  // reach blocks that were read recently; on the 6x5 lattice this made the
  // apply 3-4 % faster than ascending h (fewer neighbour blocks from DRAM)
  // (one pass over the reversed values in ascending order, each h to its class)
  std::vector<std::vector<uint32_t>> seg(t.Nlo + 1);
  for (uint32_t r = 0; r < nhi; ++r) {
    uint32_t h = 0;
    for (int b = 0; b < t.Nhi; ++b)
      if (r >> b & 1u) h |= 1u << (t.Nhi - 1 - b);
    const int k = t.n_up - popc32(h);
    if (k >= 0 && k <= t.Nlo) seg[k].push_back(h);
  }
  for (int k : ks) {
    blk.insert(blk.end(), seg[k].begin(), seg[k].end());
    while (blk.size() % kBundleMax) blk.push_back(kNoBlockEntry);
  }
}

// ---- parameter surface -------------------------------------------------------------
namespace {

struct Params {
  std::map<std::string, std::string> kv;
  bool has(const std::string& k) const { return kv.count(k) != 0; }
};

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// "KEY = value" statements separated by newlines, ';' or ','; '{' '}' task
// blocks are flattened (later assignments win); '//' starts a comment.
int parse_kv(const char* text, Params& p) {
  std::string s(text ? text : "");
  std::string cur;
  std::vector<std::string> stmts;
  bool inq = false;
  for (size_t i = 0; i < s.size(); ++i) {
    const char c = s[i];
    if (c == '"') inq = !inq;
    if (!inq && c == '/' && i + 1 < s.size() && s[i + 1] == '/') {
      while (i < s.size() && s[i] != '\n') ++i;
      stmts.push_back(cur);
      cur.clear();
      continue;
    }
    if (!inq && (c == '\n' || c == ';' || c == ',' || c == '{' || c == '}')) {
      stmts.push_back(cur);
      cur.clear();
    } else {
      cur += c;
    }
  }
  stmts.push_back(cur);
  for (auto& st : stmts) {
    const std::string t = trim(st);
    if (t.empty()) continue;
    const size_t eq = t.find('=');
    if (eq == std::string::npos) return fail(AED_ERR_INVALID, "parameter statement without '=': " + t);
    std::string key = trim(t.substr(0, eq)), val = trim(t.substr(eq + 1));
    if (val.size() >= 2 && val.front() == '"' && val.back() == '"') val = val.substr(1, val.size() - 2);
    p.kv[key] = val;
  }
  return AED_OK;
}

// Small expression evaluator: numbers, + - * / ^, parentheses, sqrt(), and
// parameter names (resolved recursively through the model defaults).
struct Eval {
  const std::map<std::string, std::string>& kv;
  const std::map<std::string, std::string>& defaults;
  int depth = 0;

  double name(const std::string& n) {
    if (++depth > 64) throw std::runtime_error("parameter recursion too deep at " + n);
    double v;
    auto it = kv.find(n);
    if (it != kv.end()) {
      v = expr_str(it->second);
    } else {
      auto d = defaults.find(n);
      if (d == defaults.end()) throw std::runtime_error("undefined parameter " + n);
      v = expr_str(d->second);
    }
    --depth;
    return v;
  }
  double expr_str(const std::string& s) {
    size_t pos = 0;
    double v = sum(s, pos);
    skip(s, pos);
    if (pos != s.size()) throw std::runtime_error("cannot evaluate '" + s + "'");
    return v;
  }
  static void skip(const std::string& s, size_t& p) {
    while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
  }
  double sum(const std::string& s, size_t& p) {
    double v = prod(s, p);
    while (true) {
      skip(s, p);
      if (p < s.size() && (s[p] == '+' || s[p] == '-')) {
        const char op = s[p++];
        const double r = prod(s, p);
        v = op == '+' ? v + r : v - r;
      } else {
        return v;
      }
    }
  }
  double prod(const std::string& s, size_t& p) {
    double v = power(s, p);
    while (true) {
      skip(s, p);
      if (p < s.size() && (s[p] == '*' || s[p] == '/')) {
        const char op = s[p++];
        const double r = power(s, p);
        v = op == '*' ? v * r : v / r;
      } else {
        return v;
      }
    }
  }
  double power(const std::string& s, size_t& p) {
    double v = unary(s, p);
    skip(s, p);
    if (p < s.size() && s[p] == '^') {
      ++p;
      v = std::pow(v, power(s, p));
    }
    return v;
  }
  double unary(const std::string& s, size_t& p) {
    skip(s, p);
    if (p < s.size() && s[p] == '-') {
      ++p;
      return -unary(s, p);
    }
    if (p < s.size() && s[p] == '+') {
      ++p;
      return unary(s, p);
    }
    return atom(s, p);
  }
  double atom(const std::string& s, size_t& p) {
    skip(s, p);
    if (p >= s.size()) throw std::runtime_error("unexpected end of expression");
    if (s[p] == '(') {
      ++p;
      const double v = sum(s, p);
      skip(s, p);
      if (p >= s.size() || s[p] != ')') throw std::runtime_error("missing ')'");
      ++p;
      return v;
    }
    if (std::isdigit((unsigned char)s[p]) || s[p] == '.') {
      size_t q = p;
      while (q < s.size() && (std::isdigit((unsigned char)s[q]) || s[q] == '.')) ++q;
      if (q < s.size() && (s[q] == 'e' || s[q] == 'E')) {
        size_t r = q + 1;
        if (r < s.size() && (s[r] == '+' || s[r] == '-')) ++r;
        if (r < s.size() && std::isdigit((unsigned char)s[r])) {
          q = r;
          while (q < s.size() && std::isdigit((unsigned char)s[q])) ++q;
        }
      }
      const double v = std::stod(s.substr(p, q - p));
      p = q;
      return v;
    }
    if (std::isalpha((unsigned char)s[p]) || s[p] == '_') {
      size_t q = p;
      while (q < s.size() && (std::isalnum((unsigned char)s[q]) || s[q] == '_' || s[q] == '\'' || s[q] == '#')) ++q;
      const std::string id = s.substr(p, q - p);
      p = q;
      skip(s, p);
      if (p < s.size() && s[p] == '(') {
        ++p;
        skip(s, p);
        if (id == "random") throw std::runtime_error("random() disorder is not supported; pass per-bond couplings");
        const double a = sum(s, p);
        skip(s, p);
        if (p >= s.size() || s[p] != ')') throw std::runtime_error("missing ')' after " + id);
        ++p;
        if (id == "sqrt") return std::sqrt(a);
        if (id == "abs") return std::fabs(a);
        throw std::runtime_error("unsupported function " + id);
      }
      return name(id);
    }
    throw std::runtime_error(std::string("unexpected character '") + s[p] + "'");
  }
};

// spin HAMILTONIAN defaults (lib/xml/models.xml.in:343-358) and BONDTERM /
// SITETERM parameter defaults (models.xml.in:360-371).
const std::map<std::string, std::string>& spin_defaults() {
  static const std::map<std::string, std::string> d = {
      {"J0", "0"},    {"J", "J0"},     {"Jz", "J"},      {"Jxy", "J"},     {"Jz0", "Jz"},
      {"Jxy0", "Jxy"}, {"J1", "0"},    {"J'", "J1"},     {"Jz'", "J'"},    {"Jxy'", "J'"},
      {"Jz1", "Jz'"}, {"Jxy1", "Jxy'"}, {"h", "0"},      {"Gamma", "0"},   {"D", "0"},
      {"K", "0"},     {"local_S", "1/2"}, {"Sz_total", "0"}};
  return d;
}

struct LatticeSpec {
  int dim;
  const char* ext_w_default;  // W default: "L" or "2" (2D only)
  bool periodic[2];
  int n_edges;
  int off_src[2][2], off_tgt[2][2], etype[2];
};

// Unit cells and finite lattices of lib/xml/lattices.xml.in (simple1d 174-177,
// complex1d 179-183, simple2d 185-189, anisotropic2d 205-209; chain 416-423,
// nnn chain 434-450, square 326-346, anisotropic square 470-479, ladder 494-516).
bool lattice_spec(const std::string& name, LatticeSpec& L) {
  std::memset(&L, 0, sizeof L);
  auto set1d = [&](bool per, int ne) {
    L.dim = 1;
    L.periodic[0] = per;
    L.n_edges = ne;
    L.off_src[0][0] = 0;
    L.off_tgt[0][0] = 1;
    L.etype[0] = 0;
    if (ne == 2) {
      L.off_src[1][0] = 0;
      L.off_tgt[1][0] = 2;
      L.etype[1] = 1;
    }
  };
  auto set2d = [&](bool p0, bool p1, bool aniso, const char* wdef) {
    L.dim = 2;
    L.periodic[0] = p0;
    L.periodic[1] = p1;
    L.ext_w_default = wdef;
    L.n_edges = 2;
    if (!aniso) {  // simple2d: (0,0)->(0,1), then (0,0)->(1,0), both type 0
      L.off_tgt[0][0] = 0; L.off_tgt[0][1] = 1; L.etype[0] = 0;
      L.off_tgt[1][0] = 1; L.off_tgt[1][1] = 0; L.etype[1] = 0;
    } else {  // anisotropic2d: type 0 (0,0)->(1,0), type 1 (0,0)->(0,1)
      L.off_tgt[0][0] = 1; L.off_tgt[0][1] = 0; L.etype[0] = 0;
      L.off_tgt[1][0] = 0; L.off_tgt[1][1] = 1; L.etype[1] = 1;
    }
  };
  if (name == "chain lattice") set1d(true, 1);
  else if (name == "open chain lattice") set1d(false, 1);
  else if (name == "nnn chain lattice") set1d(true, 2);
  else if (name == "nnn open chain lattice") set1d(false, 2);
  else if (name == "square lattice") set2d(true, true, false, "L");
  else if (name == "open square lattice") set2d(false, false, false, "L");
  else if (name == "anisotropic square lattice") set2d(true, true, true, "L");
  else if (name == "ladder") set2d(true, false, true, "2");
  else if (name == "open ladder") set2d(false, false, true, "2");
  else return false;
  return true;
}

bool flag_true(const std::string& v) { return !(v == "false" || v == "0" || v == "False" || v == "FALSE"); }

// Lattice of the parameters: its spec and extents (L, W with the lattice's
// W default).
struct Geometry {
  LatticeSpec L;
  int ext[2] = {1, 1};
  int N = 0;
};

int read_geometry(const Params& p, Eval& ev, Geometry& g) {
  auto it = p.kv.find("LATTICE");
  const std::string latname = it == p.kv.end() ? "" : it->second;
  if (!lattice_spec(latname, g.L)) return fail(AED_ERR_INVALID, "unsupported LATTICE \"" + latname + "\"");
  g.ext[0] = (int)std::lround(ev.name("L"));
  g.ext[1] = 1;
  if (g.L.dim == 2) g.ext[1] = p.has("W") ? (int)std::lround(ev.name("W")) : (int)std::lround(ev.expr_str(g.L.ext_w_default));
  if (g.ext[0] < 1 || g.ext[1] < 1) return fail(AED_ERR_INVALID, "lattice extents must be positive");
  g.N = g.ext[0] * g.ext[1];
  return AED_OK;
}

}  // namespace

int lattice_geometry(const char* text, int* dim, int ext[2], int periodic[2]) {
  Params p;
  int rc = parse_kv(text, p);
  if (rc) return rc;
  Eval ev{p.kv, spin_defaults()};
  try {
    Geometry g;
    if ((rc = read_geometry(p, ev, g))) return rc;
    *dim = g.L.dim;
    for (int d = 0; d < g.L.dim; ++d) {
      ext[d] = g.ext[d];
      periodic[d] = g.L.periodic[d] ? 1 : 0;
    }
  } catch (const std::exception& e) {
    return fail(AED_ERR_INVALID, std::string("parameter error: ") + e.what());
  }
  return AED_OK;
}

int lattice_momenta(const char* text, int* n_dirs, std::vector<std::vector<double>>& ks) {
  Params p;
  int rc = parse_kv(text, p);
  if (rc) return rc;
  Eval ev{p.kv, spin_defaults()};
  ks.clear();
  try {
    Geometry g;
    if ((rc = read_geometry(p, ev, g))) return rc;
    std::vector<int> dirs;
    for (int d = 0; d < g.L.dim; ++d)
      if (g.L.periodic[d]) dirs.push_back(d);
    *n_dirs = (int)dirs.size();
    auto tm = p.kv.find("TOTAL_MOMENTUM");
    if (tm != p.kv.end() && !tm->second.empty()) {
      // read_vector_resize (vectorio.hpp:52-60): whitespace-separated components
      std::istringstream in(tm->second);
      std::vector<double> k;
      std::string tok;
      while (in >> tok) k.push_back(ev.expr_str(tok));
      if (k.size() != dirs.size())
        return fail(AED_ERR_INVALID, "TOTAL_MOMENTUM needs one component per periodic direction (hypercubic.h:428-430)");
      ks.push_back(k);
    } else if (flag_true(p.has("TRANSLATION_SYMMETRY") ? p.kv.at("TRANSLATION_SYMMETRY") : "true")) {
      // translation_momenta (hypercubic.h:403-423): the first periodic direction slowest
      for (int d : dirs) {
        std::vector<std::vector<double>> nk;
        if (ks.empty()) {
          for (int j = 0; j < g.ext[d]; ++j) nk.push_back({2. * j * M_PI / g.ext[d]});
        } else {
          for (const auto& k : ks)
            for (int j = 0; j < g.ext[d]; ++j) {
              std::vector<double> kk = k;
              kk.push_back(2. * j * M_PI / g.ext[d]);
              nk.push_back(kk);
            }
        }
        ks.swap(nk);
      }
    }
  } catch (const std::exception& e) {
    return fail(AED_ERR_INVALID, std::string("parameter error: ") + e.what());
  }
  return AED_OK;
}

int lattice_translations(const char* text, const double* k, int n_k, int* n_sites, std::vector<int>& maps,
                         std::vector<double>& re, std::vector<double>& im) {
  Params p;
  int rc = parse_kv(text, p);
  if (rc) return rc;
  Eval ev{p.kv, spin_defaults()};
  maps.clear();
  re.clear();
  im.clear();
  try {
    Geometry g;
    if ((rc = read_geometry(p, ev, g))) return rc;
    std::vector<int> dirs;
    for (int d = 0; d < g.L.dim; ++d)
      if (g.L.periodic[d]) dirs.push_back(d);
    if (n_k != (int)dirs.size())
      return fail(AED_ERR_INVALID, "one momentum component per periodic direction (hypercubic.h:428-430)");
    *n_sites = g.N;
    // hypercubic_lattice::translations (hypercubic.h:425-464): the first
    // periodic direction fastest; translation t moves cell c to the cell at
    // c + shift (one vertex per cell for these lattices)
    std::vector<int> shift(dirs.size(), 0);
    while (true) {
      int off[2] = {0, 0};
      double phase = 0.;
      for (size_t i = 0; i < dirs.size(); ++i) {
        off[dirs[i]] = shift[i];
        phase += shift[i] * k[i];
      }
      const std::complex<double> ph = std::exp(std::complex<double>(0., phase));
      re.push_back(ph.real());
      im.push_back(ph.imag());
      for (int c = 0; c < g.N; ++c) {
        int cc[2] = {g.L.dim == 1 ? c : c / g.ext[1], g.L.dim == 1 ? 0 : c % g.ext[1]};
        for (int d = 0; d < g.L.dim; ++d) cc[d] = (cc[d] + off[d]) % g.ext[d];
        maps.push_back(g.L.dim == 1 ? cc[0] : cc[0] * g.ext[1] + cc[1]);
      }
      bool done = true;
      for (size_t i = 0; i < shift.size(); ++i) {
        if (++shift[i] >= g.ext[dirs[i]]) {
          shift[i] = 0;
        } else {
          done = false;
          break;
        }
      }
      if (done) break;
    }
  } catch (const std::exception& e) {
    return fail(AED_ERR_INVALID, std::string("parameter error: ") + e.what());
  }
  return AED_OK;
}

int parse_parameters(const char* text, ParsedParams& out, const GraphSpec* graph) {
  Params p;
  int rc = parse_kv(text, p);
  if (rc) return rc;
  out = ParsedParams();
  std::memset(&out.info, 0, sizeof out.info);
  Eval ev{p.kv, spin_defaults()};
  try {
    auto str = [&](const std::string& k, const std::string& dflt) {
      auto it = p.kv.find(k);
      return it == p.kv.end() ? dflt : it->second;
    };
    const std::string model = str("MODEL", "");
    if (model != "spin") return fail(AED_ERR_INVALID, "MODEL must be \"spin\" (got \"" + model + "\")");
    const double spin = ev.name("local_S");
    const int two_s = (int)std::lround(2.0 * spin);
    if (std::fabs(2.0 * spin - two_s) > 1e-12 || two_s < 1 || two_s > 4)
      return fail(AED_ERR_INVALID, "local_S must be one of 1/2, 1, 3/2, 2");
    const std::string latname = str("LATTICE", "");
    LatticeSpec L;
    if (!graph && !lattice_spec(latname, L))
      return fail(AED_ERR_INVALID, "unsupported LATTICE \"" + latname + "\"");
    const std::string cq = str("CONSERVED_QUANTUMNUMBERS", "");
    if (cq.find("Sz") == std::string::npos)
      return fail(AED_ERR_INVALID, "CONSERVED_QUANTUMNUMBERS must contain Sz (full Hilbert space not supported)");
    if (!p.has("Sz_total"))
      return fail(AED_ERR_INVALID, "Sz_total must be given (one sector per handle; alps_b200.sparsediag loops over them)");
    // the graph: edges (source, target, type) in graph order and the type of every vertex
    std::vector<int> esrc, etgt, etyp, vtyp;
    int N = 0;
    if (graph) {
      N = graph->n;
      if (N < 2 || N > 32) return fail(AED_ERR_INVALID, "number of sites must be in 2..32");
      if ((int)graph->vtype.size() != N) return fail(AED_ERR_INVALID, "one type per vertex expected");
      vtyp = graph->vtype;
      for (size_t e = 0; e < graph->src.size(); ++e) {
        const int si = graph->src[e], ti = graph->tgt[e];
        if (si < 0 || si >= N || ti < 0 || ti >= N) return fail(AED_ERR_INVALID, "edge vertex out of range");
        if (si == ti) return fail(AED_ERR_INVALID, "an edge joins a vertex to itself");
        if (graph->etype[e] < 0) return fail(AED_ERR_INVALID, "negative edge type");
        esrc.push_back(si);
        etgt.push_back(ti);
        etyp.push_back(graph->etype[e]);
      }
      for (int t : vtyp)
        if (t < 0) return fail(AED_ERR_INVALID, "negative vertex type");
    } else {
      const int Lx = (int)std::lround(ev.name("L"));
      int Wy = 1;
      if (L.dim == 2) Wy = p.has("W") ? (int)std::lround(ev.name("W")) : (int)std::lround(ev.expr_str(L.ext_w_default));
      if (Lx < 1 || Wy < 1) return fail(AED_ERR_INVALID, "lattice extents must be positive");
      N = Lx * Wy;
      if (N < 2 || N > 32) return fail(AED_ERR_INVALID, "number of sites must be in 2..32");
      // edges: cell by cell (last coordinate fastest), unit-cell edge order,
      // open boundaries drop edges, self-loops are dropped (latticegraph.h:98-136)
      const int ext[2] = {Lx, Wy};
      for (int c = 0; c < N; ++c) {
        int cc[2];
        if (L.dim == 1) {
          cc[0] = c;
          cc[1] = 0;
        } else {
          cc[0] = c / Wy;
          cc[1] = c % Wy;
        }
        for (int e = 0; e < L.n_edges; ++e) {
          int src[2], tgt[2];
          bool ok = true;
          for (int d = 0; d < L.dim; ++d) {
            src[d] = cc[d] + L.off_src[e][d];
            tgt[d] = cc[d] + L.off_tgt[e][d];
            for (int* v : {&src[d], &tgt[d]}) {
              if (*v < 0 || *v >= ext[d]) {
                if (!L.periodic[d]) ok = false;
                *v = ((*v % ext[d]) + ext[d]) % ext[d];
              }
            }
          }
          if (!ok) continue;
          const int si = L.dim == 1 ? src[0] : src[0] * Wy + src[1];
          const int ti = L.dim == 1 ? tgt[0] : tgt[0] * Wy + tgt[1];
          if (si == ti) continue;
          esrc.push_back(si);
          etgt.push_back(ti);
          etyp.push_back(L.etype[e]);
        }
      }
      vtyp.assign(N, 0);  // the supported lattices have one site type
    }
    // the sector's digit sum Sz_total + N S (spin 1/2: the number of up spins)
    const double szt = ev.name("Sz_total");
    const double nup_d = N * two_s / 2.0 + szt;
    const int n_up = (int)std::lround(nup_d);
    if (std::fabs(nup_d - n_up) > 1e-9 || n_up < 0 || n_up > N * two_s)
      return fail(AED_ERR_INVALID, "Sz_total incompatible with the number of sites");
    {
      for (size_t e = 0; e < esrc.size(); ++e) {
        const int si = esrc[e], ti = etgt[e];
        const std::string t = std::to_string(etyp[e]);
        // Jz# / Jxy# / K#: HAMILTONIAN parameters first, then BONDTERM default J#
        auto coupling = [&](const std::string& base) {
          const std::string n = base + t;
          if (p.has(n) || spin_defaults().count(n)) return ev.name(n);
          const std::string j = "J" + t;
          if (p.has(j) || spin_defaults().count(j)) return ev.name(j);
          return 0.0;
        };
        const double jz = coupling("Jz"), jxy = coupling("Jxy");
        // K# has BONDTERM default 0 (models.xml.in:370); the HAMILTONIAN-level K
        // is not substituted into it
        const std::string kn = "K" + t;
        const double kq = p.has(kn) ? ev.name(kn) : 0.0;
        if ((int)out.s1.size() >= kMaxBonds) return fail(AED_ERR_INVALID, "too many bonds");
        out.s1.push_back(si);
        out.s2.push_back(ti);
        out.jz.push_back(jz);
        out.jxy.push_back(jxy);
        out.kq.push_back(kq);
      }
    }
    // site terms of vertex type t: h# = h, D# = D, Gamma# = Gamma (SITETERM
    // defaults, models.xml.in:360-365)
    std::vector<double> sh(N), sd(N);
    bool any_site = false;
    for (int i = 0; i < N; ++i) {
      const std::string t = std::to_string(vtyp[i]);
      const double h = p.has("h" + t) ? ev.name("h" + t) : ev.name("h");
      const double d = p.has("D" + t) ? ev.name("D" + t) : ev.name("D");
      const double g = p.has("Gamma" + t) ? ev.name("Gamma" + t) : ev.name("Gamma");
      if (g != 0.0) return fail(AED_ERR_INVALID, "Gamma (transverse field) breaks Sz conservation");
      sh[i] = h;
      sd[i] = d;
      any_site = any_site || h != 0.0 || d != 0.0;
    }
    if (any_site) {
      out.site_h = sh;
      out.site_d = sd;
      out.info.has_site_terms = 1;
    }
    out.info.n_sites = N;
    out.info.n_up = n_up;
    out.info.two_s = two_s;
    out.info.n_bonds = (int)out.s1.size();
    out.info.number_eigenvalues = p.has("NUMBER_EIGENVALUES") ? (int)std::lround(ev.name("NUMBER_EIGENVALUES")) : 1;
    out.info.max_iterations = p.has("MAX_ITERATIONS") ? (int)std::lround(ev.name("MAX_ITERATIONS")) : 0;
    if (out.info.number_eigenvalues < 1) return fail(AED_ERR_INVALID, "NUMBER_EIGENVALUES must be >= 1");
  } catch (const std::exception& e) {
    return fail(AED_ERR_INVALID, std::string("parameter error: ") + e.what());
  }
  return AED_OK;
}

}  // namespace aed
