/* Test-infrastructure shim: boost::generator_iterator over a generator.
 * Like Boost's, it draws one value on construction and one per increment. */
#ifndef ORACLE_SHIM_BOOST_GENERATOR_ITERATOR_HPP
#define ORACLE_SHIM_BOOST_GENERATOR_ITERATOR_HPP
namespace boost {
template <typename Gen>
class generator_iterator {
 public:
  typedef typename Gen::result_type value_type;
  explicit generator_iterator(Gen *g) : g_(g), v_((*g)()) {}
  value_type operator*() const { return v_; }
  generator_iterator &operator++() { v_ = (*g_)(); return *this; }
  generator_iterator operator++(int) { generator_iterator t(*this); v_ = (*g_)(); return t; }
 private:
  Gen *g_;
  value_type v_;
};
}  // namespace boost
#endif
