/* Test-infrastructure shim: boost::variate_generator<Engine&, Dist>. */
#ifndef ORACLE_SHIM_BOOST_VARIATE_GENERATOR_HPP
#define ORACLE_SHIM_BOOST_VARIATE_GENERATOR_HPP
#include <type_traits>
namespace boost {
template <typename EngineRef, typename Dist>
class variate_generator {
 public:
  typedef typename Dist::result_type result_type;
  variate_generator(EngineRef e, Dist d) : eng_(e), dist_(d) {}
  result_type operator()() { return dist_(eng_); }
 private:
  EngineRef eng_;
  Dist dist_;
};
}  // namespace boost
#endif
