/* Test-infrastructure shim: boost::function2<R,A,B> as std::function. */
#ifndef ORACLE_SHIM_BOOST_FUNCTION_HPP
#define ORACLE_SHIM_BOOST_FUNCTION_HPP
#include <functional>
namespace boost {
template <typename R, typename A, typename B>
class function2 : public std::function<R(A, B)> {
 public:
  template <typename F>
  function2(F f) : std::function<R(A, B)>(f) {}
};
}  // namespace boost
#endif
