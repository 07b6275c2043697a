/* Test-infrastructure shim: a minimal stand-in for boost::format so the
 * reference sources compile without Boost.  The oracle silences the
 * reference logger, so these objects are built but never rendered in a
 * hot loop; they still format "%d %f %e %s"-style strings faithfully
 * enough for debugging. */
#ifndef ORACLE_SHIM_BOOST_FORMAT_HPP
#define ORACLE_SHIM_BOOST_FORMAT_HPP
#include <sstream>
#include <string>
#include <ostream>
namespace boost {
class format {
 public:
  explicit format(const char *f) : fmt_(f ? f : ""), pos_(0) {}
  explicit format(const std::string &f) : fmt_(f), pos_(0) {}
  template <typename T>
  format &operator%(const T &v) {
    std::size_t p = fmt_.find('%', pos_);
    while (p != std::string::npos && p + 1 < fmt_.size() && fmt_[p + 1] == '%') p = fmt_.find('%', p + 2);
    std::ostringstream os;
    os << v;
    if (p == std::string::npos) { fmt_ += " " + os.str(); pos_ = fmt_.size(); return *this; }
    std::size_t e = p + 1;
    while (e < fmt_.size() && std::string("diouxXeEfFgGaAcsp").find(fmt_[e]) == std::string::npos) e++;
    fmt_.replace(p, e - p + 1, os.str());
    pos_ = p + os.str().size();
    return *this;
  }
  std::string str() const { return fmt_; }
  friend std::ostream &operator<<(std::ostream &os, const format &f) { return os << f.fmt_; }
 private:
  std::string fmt_;
  std::size_t pos_;
};
}  // namespace boost
#endif
