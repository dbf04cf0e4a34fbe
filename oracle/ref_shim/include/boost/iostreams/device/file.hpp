/* boost/iostreams/device/file.hpp — see filtering_stream.hpp (oracle shim only). */
#ifndef PLATO_ORACLE_SHIM_BOOST_FILE_HPP
#define PLATO_ORACLE_SHIM_BOOST_FILE_HPP
#include <string>
#include "boost/iostreams/filtering_stream.hpp"
namespace boost {
namespace iostreams {
struct file_source { explicit file_source(const std::string&, std::ios_base::openmode = std::ios_base::in) {} };
struct file_sink { explicit file_sink(const std::string&, std::ios_base::openmode = std::ios_base::out) {} };
}  // namespace iostreams
}  // namespace boost
#endif
