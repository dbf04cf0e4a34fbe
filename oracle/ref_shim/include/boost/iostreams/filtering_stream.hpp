/* boost/iostreams/filtering_stream.hpp — for the oracle shim (test
 * infrastructure only): stream types the reference's file helpers name.
 * The shim builds its graphs in memory and reads or writes no file through
 * them; push() accepts any filter or device and ignores it. */
#ifndef PLATO_ORACLE_SHIM_BOOST_FILTERING_STREAM_HPP
#define PLATO_ORACLE_SHIM_BOOST_FILTERING_STREAM_HPP
#include <cstdint>
#include <ios>
#include <iostream>
#include <sstream>
#include <string>
namespace boost {
namespace iostreams {
typedef int64_t stream_offset;
struct source_tag {};
struct sink_tag {};
struct closable_tag {};
struct multichar_tag {};
struct seekable_device_tag {};
struct bidirectional_device_tag {};
struct input_seekable {};
struct input {};
struct output {};
template <typename Mode, typename Ch = char>
class filtering_stream : public std::stringstream {
 public:
  template <typename T> void push(const T&, std::streamsize = 0, std::streamsize = 0) {}
  void reset() {}
  bool empty() const { return true; }
};
class filtering_istream : public std::istringstream {
 public:
  template <typename T> void push(const T&, std::streamsize = 0, std::streamsize = 0) {}
  void reset() {}
  bool empty() const { return true; }
};
class filtering_ostream : public std::ostringstream {
 public:
  template <typename T> void push(const T&, std::streamsize = 0, std::streamsize = 0) {}
  void reset() {}
  bool empty() const { return true; }
};
}  // namespace iostreams
}  // namespace boost
#endif
