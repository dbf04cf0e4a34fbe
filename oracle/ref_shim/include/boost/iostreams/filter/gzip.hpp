/* boost/iostreams/filter/gzip.hpp — see filtering_stream.hpp (oracle shim only). */
#ifndef PLATO_ORACLE_SHIM_BOOST_GZIP_HPP
#define PLATO_ORACLE_SHIM_BOOST_GZIP_HPP
#include "boost/iostreams/filtering_stream.hpp"
namespace boost {
namespace iostreams {
struct gzip_params { explicit gzip_params(int = 0) {} };
struct gzip_decompressor { gzip_decompressor() {} };
struct gzip_compressor { explicit gzip_compressor(gzip_params = gzip_params()) {} };
namespace gzip { constexpr int best_speed = 1, best_compression = 9, default_compression = 6; }
}  // namespace iostreams
}  // namespace boost
#endif
