/* boost/iostreams/stream.hpp — see filtering_stream.hpp (oracle shim only). */
#ifndef PLATO_ORACLE_SHIM_BOOST_STREAM_HPP
#define PLATO_ORACLE_SHIM_BOOST_STREAM_HPP
#include "boost/iostreams/filtering_stream.hpp"
namespace boost {
namespace iostreams {
template <typename Device>
class stream : public std::stringstream {
 public:
  stream() {}
  template <typename... A> explicit stream(A&&...) {}
  template <typename... A> void open(A&&...) {}
  bool is_open() const { return false; }
};
}  // namespace iostreams
}  // namespace boost
#endif
