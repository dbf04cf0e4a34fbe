/* boost/align.hpp — align_up for the oracle shim (test infrastructure only). */
#ifndef PLATO_ORACLE_SHIM_BOOST_ALIGN_HPP
#define PLATO_ORACLE_SHIM_BOOST_ALIGN_HPP
#include <cstddef>
namespace boost {
namespace alignment {
inline std::size_t align_up(std::size_t v, std::size_t a) { return (v + a - 1) / a * a; }
inline std::size_t align_down(std::size_t v, std::size_t a) { return v / a * a; }
}  // namespace alignment
}  // namespace boost
#endif
