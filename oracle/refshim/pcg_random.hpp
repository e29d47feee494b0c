/* Stand-in for the un-vendored pcg-cpp header that the reference's rng.h includes.
 * The reference uses it only to fill random test vectors (_RNG::randu32); none of the
 * arithmetic on the prover path touches it.  This stub is a plain 32-bit LCG with the
 * two entry points rng.cpp needs (construct/seed from an integer or a seed sequence,
 * and operator() returning 32 bits).  It is test infrastructure for building the
 * reference CPU library as an oracle, never part of the product. */
#ifndef CUSNARKS_B200_PCG_STUB_HPP
#define CUSNARKS_B200_PCG_STUB_HPP
#include <cstdint>
#include <random>

namespace pcg_extras {
template <typename Source>
struct seed_seq_from {
  uint64_t value;
  seed_seq_from() { Source s; value = ((uint64_t)s() << 32) ^ (uint64_t)s(); }
};
}  // namespace pcg_extras

class pcg32 {
 public:
  explicit pcg32(uint64_t seed = 42u) : state_(seed * 6364136223846793005ull + 1442695040888963407ull) {}
  void seed(uint64_t s) { state_ = s * 6364136223846793005ull + 1442695040888963407ull; }
  template <typename Source>
  void seed(const pcg_extras::seed_seq_from<Source>& s) { seed(s.value); }
  uint32_t operator()() {
    state_ = state_ * 6364136223846793005ull + 1442695040888963407ull;
    return (uint32_t)(state_ >> 33);
  }
 private:
  uint64_t state_;
};
#endif
