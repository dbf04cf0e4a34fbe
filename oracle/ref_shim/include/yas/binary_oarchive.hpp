/* yas/binary_oarchive.hpp — the reference serialises trivial message types
 * by memcpy and only non-trivial ones through yas; the engine path sends only
 * trivial messages (the file-list shuffle of its path helpers is the only
 * non-trivial user, and the shim reads no files), so for the oracle shim
 * (test infrastructure only) these archives exist to be compiled and abort
 * if ever used. */
#ifndef PLATO_ORACLE_SHIM_YAS_OARCHIVE_HPP
#define PLATO_ORACLE_SHIM_YAS_OARCHIVE_HPP
#include <cstddef>
#include <cstdio>
#include <cstdlib>
namespace yas {
inline void plato_shim_unused(const char* what) {
  std::fprintf(stderr, "oracle shim: %s is not available\n", what);
  std::abort();
}
enum options : std::size_t { binary = 1, text = 2, json = 4, ehost = 8, elittle = 16, ebig = 32, no_header = 64 };
template <typename OS, std::size_t F>
struct binary_oarchive {
  explicit binary_oarchive(OS&) {}
  template <typename T> binary_oarchive& operator&(const T&) {
    plato_shim_unused("yas serialisation");
    return *this;
  }
};
}  // namespace yas
#endif
