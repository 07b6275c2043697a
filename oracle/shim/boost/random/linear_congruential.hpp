/* Test-infrastructure shim for Boost.Random 1.61 minstd_rand:
 * x_{n+1} = 48271 * x_n mod (2^31 - 1), seed 0 mapped to 1 as Boost does.
 * Restated from the published Park-Miller "minimal standard" definition. */
#ifndef ORACLE_SHIM_BOOST_LCG_HPP
#define ORACLE_SHIM_BOOST_LCG_HPP
#include <cstdint>
namespace boost {
class minstd_rand {
 public:
  typedef std::int32_t result_type;
  explicit minstd_rand(std::int64_t seed = 1) { this->seed(seed); }
  void seed(std::int64_t s) {
    std::int64_t m = 2147483647;
    s %= m;
    if (s < 0) s += m;
    x_ = (s == 0) ? 1 : s;
  }
  result_type operator()() {
    x_ = (x_ * 48271) % 2147483647;
    return static_cast<result_type>(x_);
  }
  static result_type min() { return 1; }
  static result_type max() { return 2147483646; }
 private:
  std::int64_t x_;
};
}  // namespace boost
#endif
