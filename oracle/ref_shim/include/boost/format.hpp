/* boost/format.hpp — message formatting for the reference's log and error
 * text, for the oracle shim (test infrastructure only): the format string
 * followed by its arguments. */
#ifndef PLATO_ORACLE_SHIM_BOOST_FORMAT_HPP
#define PLATO_ORACLE_SHIM_BOOST_FORMAT_HPP
#include <ostream>
#include <sstream>
#include <string>
namespace boost {
class format {
 public:
  explicit format(const std::string& f) { os_ << f; }
  template <typename T> format& operator%(const T& v) {
    os_ << " " << v;
    return *this;
  }
  std::string str() const { return os_.str(); }
 private:
  std::ostringstream os_;
};
inline std::ostream& operator<<(std::ostream& os, const format& f) { return os << f.str(); }
}  // namespace boost
#endif
