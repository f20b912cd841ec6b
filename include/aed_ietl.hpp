// aed_ietl.hpp -- drop-in MATRIX / VS types for ietl::lanczos over libaed.so.
//
// ietl::lanczos<MATRIX, VS> (src/ietl/lanczos.h:64-119 of the ALPS tree) needs
// a matrix type, a vector space (src/ietl/vectorspace.h:23-46) and the free
// functions mult, dot, two_norm, generate, clear, copy found in namespace ietl
// (src/ietl/interface/ublas.h:27-63), plus vector algebra v *= s, v /= s,
// v -= s*w, v += s*w, v = s*w, deep copies and an O(1) std::swap
// (lanczos.h:383-404).  This header provides all of them on device vectors
// owned by the engine:
//
//   aed_ietl::matrix H(model_desc);                 // the Hamiltonian handle
//   aed_ietl::vectorspace vs(H);
//   ietl::lanczos<aed_ietl::matrix, aed_ietl::vectorspace> lanczos(H, vs);
//   ietl::lanczos_iteration_nlowest<double> iter(max_iter, n);
//   lanczos.calculate_eigenvalues(iter, aed_ietl::seeded_generator{seed});
//
// Every operation returns only after the device work it queued has been
// ordered on the handle's stream; scalar results (dot, two_norm) synchronise.
// Errors throw std::runtime_error with the engine's message, as the
// reference's code expects from failures (tmatrix.h:144-145, lanczos.h:250).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "aed.h"

namespace aed_ietl {

inline void check(int rc) {
  if (rc != AED_OK) throw std::runtime_error(std::string("aed: ") + aed_last_error());
}

// MATRIX: one Sz sector of a spin-1/2 model on one GPU.
class matrix {
 public:
  explicit matrix(const aed_model_desc& m, int precision = AED_FP64, int device = 0) {
    check(aed_create(&m, precision, device, &h_));
  }
  ~matrix() {
    if (h_) aed_destroy(h_);
  }
  matrix(const matrix&) = delete;
  matrix& operator=(const matrix&) = delete;
  aed_handle* handle() const { return h_; }
  std::size_t dimension() const {
    int64_t d = 0;
    check(aed_dimension(h_, &d));
    return (std::size_t)d;
  }

 private:
  aed_handle* h_ = nullptr;
};

class vector;

// s * v, as written in lanczos.h (vec2 -= a*startvector)
struct scaled {
  double s;
  const vector& v;
};

// vector_type: a device vector with value semantics.
class vector {
 public:
  typedef double value_type;
  typedef std::size_t size_type;

  vector() = default;
  explicit vector(aed_handle* h) : h_(h) { check(aed_vec_alloc(h_, &p_)); }
  vector(const vector& o) : h_(o.h_) {
    if (h_) {
      check(aed_vec_alloc(h_, &p_));
      check(aed_vec_copy(h_, o.p_, p_));
    }
  }
  vector(vector&& o) noexcept : h_(o.h_), p_(o.p_) {
    o.h_ = nullptr;
    o.p_ = nullptr;
  }
  vector& operator=(const vector& o) {
    if (this == &o) return *this;
    if (!p_ || h_ != o.h_) {
      release();
      h_ = o.h_;
      if (h_) check(aed_vec_alloc(h_, &p_));
    }
    if (h_) check(aed_vec_copy(h_, o.p_, p_));
    return *this;
  }
  vector& operator=(vector&& o) noexcept {
    std::swap(h_, o.h_);
    std::swap(p_, o.p_);
    return *this;
  }
  ~vector() { release(); }

  vector& operator*=(double s) {
    check(aed_scal(h_, s, p_));
    return *this;
  }
  vector& operator/=(double s) {
    check(aed_div(h_, s, p_));
    return *this;
  }
  vector& operator-=(const scaled& x) {
    check(aed_axpy(h_, -x.s, x.v.p_, p_));
    return *this;
  }
  vector& operator+=(const scaled& x) {
    check(aed_axpy(h_, x.s, x.v.p_, p_));
    return *this;
  }
  vector& operator+=(const vector& x) {
    check(aed_axpy(h_, 1.0, x.p_, p_));
    return *this;
  }
  vector& operator=(const scaled& x) {
    if (!p_) {
      h_ = x.v.h_;
      check(aed_vec_alloc(h_, &p_));
    }
    check(aed_vec_copy(h_, x.v.p_, p_));
    check(aed_scal(h_, x.s, p_));
    return *this;
  }

  size_type size() const {
    int64_t d = 0;
    if (h_) check(aed_dimension(h_, &d));
    return (size_type)d;
  }
  aed_handle* handle() const { return h_; }
  void* data() const { return p_; }
  std::vector<double> to_host() const {
    std::vector<double> out(size());
    check(aed_vec_download(h_, p_, out.data()));
    return out;
  }
  void from_host(const std::vector<double>& v) { check(aed_vec_upload(h_, p_, v.data())); }

 private:
  void release() {
    if (p_ && h_) aed_vec_free(h_, p_);
    p_ = nullptr;
  }
  aed_handle* h_ = nullptr;
  void* p_ = nullptr;
};

inline scaled operator*(double s, const vector& v) { return scaled{s, v}; }

// VS: the vector space of a matrix (ietl::vectorspace semantics).
class vectorspace {
 public:
  typedef aed_ietl::vector vector_type;
  typedef double scalar_type;
  typedef std::size_t size_type;
  explicit vectorspace(const matrix& m) : h_(m.handle()), n_(m.dimension()) {}
  size_type vec_dimension() const { return n_; }
  vector_type new_vector() const { return vector_type(h_); }  // zeroed
  void project(vector_type&) const {}

 private:
  aed_handle* h_;
  size_type n_;
};

// Start-vector generator filled on the device (splitmix64 stream of `seed`):
// the engine's replacement for the host-side boost generator of sparsediag.h:98.
struct seeded_generator {
  uint64_t seed = 0;
};

}  // namespace aed_ietl

namespace ietl {

inline void mult(const aed_ietl::matrix& m, const aed_ietl::vector& x, aed_ietl::vector& y) {
  aed_ietl::check(aed_mult(m.handle(), x.data(), y.data()));
}

inline double dot(const aed_ietl::vector& x, const aed_ietl::vector& y) {
  double r = 0.0;
  aed_ietl::check(aed_dot(x.handle(), x.data(), y.data(), &r));
  return r;
}

inline double two_norm(const aed_ietl::vector& x) {
  double r = 0.0;
  aed_ietl::check(aed_nrm2(x.handle(), x.data(), &r));
  return r;
}

inline void clear(aed_ietl::vector& x) { aed_ietl::check(aed_vec_clear(x.handle(), x.data())); }

inline void copy(const aed_ietl::vector& x, aed_ietl::vector& y) { y = x; }

inline void generate(aed_ietl::vector& x, const aed_ietl::seeded_generator& g) {
  aed_ietl::check(aed_vec_fill_random(x.handle(), x.data(), g.seed));
}
inline void generate(aed_ietl::vector& x, aed_ietl::seeded_generator& g) {
  generate(x, static_cast<const aed_ietl::seeded_generator&>(g));
}

// Host generators (e.g. boost::lagged_fibonacci607): drawn on the host in
// index order from a copy of the generator, as std::generate does in
// src/ietl/interface/ublas.h:27-30, then uploaded.
template <class Gen>
inline void generate(aed_ietl::vector& x, const Gen& gen) {
  Gen g = gen;
  std::vector<double> h(x.size());
  for (auto& v : h) v = g();
  x.from_host(h);
}

}  // namespace ietl
