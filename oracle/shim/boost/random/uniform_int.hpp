/* Test-infrastructure shim for boost::uniform_int<> (Boost.Random 1.61).
 * Boost maps an engine draw to [lo, hi] by integer bucketing: with
 * brange = engine max - min and range = hi - lo < brange, it uses
 * bucket = (brange + 1) / (range + 1) and rejects results above range.
 * Restated from the published Boost.Random algorithm description. */
#ifndef ORACLE_SHIM_BOOST_UNIFORM_INT_HPP
#define ORACLE_SHIM_BOOST_UNIFORM_INT_HPP
#include <cstdint>
namespace boost {
template <typename IntType = int>
class uniform_int {
 public:
  typedef IntType result_type;
  uniform_int(IntType lo = 0, IntType hi = 9) : lo_(lo), hi_(hi) {}
  template <typename Engine>
  result_type operator()(Engine &eng) {
    std::uint64_t range = static_cast<std::uint64_t>(hi_ - lo_);
    std::uint64_t bmin = static_cast<std::uint64_t>(Engine::min());
    std::uint64_t brange = static_cast<std::uint64_t>(Engine::max()) - bmin;
    if (range == 0) return lo_;
    std::uint64_t bucket = (brange + 1) / (range + 1);
    for (;;) {
      std::uint64_t r = (static_cast<std::uint64_t>(eng()) - bmin) / bucket;
      if (r <= range) return static_cast<result_type>(r + lo_);
    }
  }
 private:
  IntType lo_, hi_;
};
}  // namespace boost
#endif
