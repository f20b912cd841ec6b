// ietl_adaptor_check.cpp -- drives include/aed_ietl.hpp the way ietl::lanczos does.
//
// The first steps of ietl::lanczos (make_first_step / make_step,
// src/ietl/lanczos.h:377-406 of the ALPS tree) are written out below with the
// same expressions on aed_ietl types, so the adaptor is exercised exactly as
// the template would exercise it.  Prints "alpha beta" per step for the test
// to compare with the oracle.  Usage: ietl_adaptor_check L steps seed
#include <cstdio>
#include <cstdlib>
#include <utility>
#include <vector>

#include "aed_ietl.hpp"

namespace {

template <class MATRIX, class VS, class GEN>
std::pair<double, double> first_step(const MATRIX& matrix_, const VS& vecspace_, typename VS::vector_type& startvector,
                                     typename VS::vector_type& vec2, GEN gen) {
  double a, b;
  ietl::generate(startvector, gen);
  vecspace_.project(startvector);
  startvector /= ietl::two_norm(startvector);
  ietl::mult(matrix_, startvector, vec2);
  a = ietl::dot(startvector, vec2);
  vec2 -= a * startvector;
  b = ietl::two_norm(vec2);
  vec2 /= b;
  return std::make_pair(a, b);
}

template <class MATRIX, class V>
std::pair<double, double> step(const MATRIX& matrix_, V& startvector, V& vec2, V& vec3, double bprev) {
  double a, b;
  b = bprev;
  ietl::mult(matrix_, vec2, vec3);
  a = ietl::dot(vec2, vec3);
  vec3 -= a * vec2;
  vec3 -= b * startvector;
  b = ietl::two_norm(vec3);
  vec3 /= b;
  std::swap(vec2, startvector);
  std::swap(vec3, vec2);
  return std::make_pair(a, b);
}

}  // namespace

int main(int argc, char** argv) {
  const int L = argc > 1 ? std::atoi(argv[1]) : 16;
  const int steps = argc > 2 ? std::atoi(argv[2]) : 20;
  const unsigned long long seed = argc > 3 ? std::strtoull(argv[3], nullptr, 10) : 1;
  std::vector<int32_t> s1, s2;
  std::vector<double> j;
  for (int i = 0; i < L; ++i) {
    s1.push_back(i);
    s2.push_back((i + 1) % L);
    j.push_back(1.0);
  }
  aed_model_desc m{L, L / 2, L, s1.data(), s2.data(), j.data(), j.data(), nullptr, nullptr, nullptr};
  try {
    aed_ietl::matrix H(m);
    aed_ietl::vectorspace vs(H);
    aed_ietl::vector startvector = vs.new_vector(), vec2 = vs.new_vector(), vec3 = vs.new_vector();
    auto ab = first_step(H, vs, startvector, vec2, aed_ietl::seeded_generator{seed});
    std::printf("%.17g %.17g\n", ab.first, ab.second);
    double b = ab.second;
    for (int k = 1; k < steps; ++k) {
      ab = step(H, startvector, vec2, vec3, b);
      b = ab.second;
      std::printf("%.17g %.17g\n", ab.first, ab.second);
    }
    // deep copy and value semantics
    aed_ietl::vector c = vec2;
    c *= 2.0;
    const double r = ietl::dot(c, vec2) / ietl::dot(vec2, vec2);
    if (r < 1.999999 || r > 2.000001) {
      std::fprintf(stderr, "copy semantics broken: %g\n", r);
      return 2;
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
