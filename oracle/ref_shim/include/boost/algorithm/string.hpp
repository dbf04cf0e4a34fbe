/* boost/algorithm/string.hpp — the prefix/suffix tests the reference's path
 * helpers use, for the oracle shim (test infrastructure only). */
#ifndef PLATO_ORACLE_SHIM_BOOST_ALGO_STRING_HPP
#define PLATO_ORACLE_SHIM_BOOST_ALGO_STRING_HPP
#include <cctype>
#include <string>
#include <vector>
namespace boost {
namespace algorithm {
inline bool starts_with(const std::string& s, const std::string& p) { return s.compare(0, p.size(), p) == 0; }
inline bool ends_with(const std::string& s, const std::string& p) {
  return s.size() >= p.size() && s.compare(s.size() - p.size(), p.size(), p) == 0;
}
inline std::string plato_shim_lower(std::string s) {
  for (auto& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  return s;
}
inline bool istarts_with(const std::string& s, const std::string& p) {
  return starts_with(plato_shim_lower(s), plato_shim_lower(p));
}
inline bool iends_with(const std::string& s, const std::string& p) {
  return ends_with(plato_shim_lower(s), plato_shim_lower(p));
}
}  // namespace algorithm
using algorithm::ends_with;
using algorithm::iends_with;
using algorithm::istarts_with;
using algorithm::starts_with;
}  // namespace boost
#endif
