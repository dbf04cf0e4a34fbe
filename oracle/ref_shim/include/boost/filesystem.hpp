/* boost/filesystem.hpp — the file-system queries the reference's path
 * helpers name, for the oracle shim (test infrastructure only), over
 * std::filesystem.  The shim builds its graphs in memory and opens no path. */
#ifndef PLATO_ORACLE_SHIM_BOOST_FILESYSTEM_HPP
#define PLATO_ORACLE_SHIM_BOOST_FILESYSTEM_HPP
#include <cstdint>
#include <filesystem>
#include <string>
namespace boost {
namespace filesystem {
using std::filesystem::directory_iterator;
using std::filesystem::path;
using std::filesystem::space;
using std::filesystem::space_info;
using std::filesystem::remove;
inline bool is_directory(const std::string& p) { return std::filesystem::is_directory(p); }
inline bool exists(const std::string& p) { return std::filesystem::exists(p); }
inline std::uintmax_t file_size(const std::string& p) { return std::filesystem::file_size(p); }
inline bool create_directories(const std::string& p) { return std::filesystem::create_directories(p); }
inline std::uintmax_t remove_all(const std::string& p) { return std::filesystem::remove_all(p); }
}  // namespace filesystem
}  // namespace boost
#endif
