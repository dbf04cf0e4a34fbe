/* yas/binary_iarchive.hpp — see binary_oarchive.hpp (oracle shim only). */
#ifndef PLATO_ORACLE_SHIM_YAS_IARCHIVE_HPP
#define PLATO_ORACLE_SHIM_YAS_IARCHIVE_HPP
#include "yas/binary_oarchive.hpp"
namespace yas {
template <typename IS, std::size_t F>
struct binary_iarchive {
  explicit binary_iarchive(IS&) {}
  template <typename T> binary_iarchive& operator&(T&) {
    plato_shim_unused("yas serialisation");
    return *this;
  }
  bool empty() const { return true; }
};
}  // namespace yas
#endif
