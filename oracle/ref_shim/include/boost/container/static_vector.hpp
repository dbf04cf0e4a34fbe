/* boost/container/static_vector.hpp — for the oracle shim (test
 * infrastructure only): a std::vector stands in for the bounded vector. */
#ifndef PLATO_ORACLE_SHIM_BOOST_STATIC_VECTOR_HPP
#define PLATO_ORACLE_SHIM_BOOST_STATIC_VECTOR_HPP
#include <cstddef>
#include <vector>
namespace boost {
namespace container {
template <typename T, std::size_t N>
class static_vector : public std::vector<T> {
 public:
  using std::vector<T>::vector;
};
}  // namespace container
}  // namespace boost
#endif
