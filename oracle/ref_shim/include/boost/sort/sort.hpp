/* boost/sort/sort.hpp — pdqsort for the oracle shim (test infrastructure
 * only).  The reference sorts with a strict total order (rank descending,
 * then id ascending, plato/algo/trustrank/trustrank.hpp:108-112), so any
 * correct sort gives the same sequence; std::sort stands in. */
#ifndef PLATO_ORACLE_SHIM_BOOST_SORT_HPP
#define PLATO_ORACLE_SHIM_BOOST_SORT_HPP
#include <algorithm>
namespace boost {
namespace sort {
template <typename It, typename Cmp> void pdqsort(It first, It last, Cmp cmp) { std::sort(first, last, cmp); }
template <typename It> void pdqsort(It first, It last) { std::sort(first, last); }
}  // namespace sort
}  // namespace boost
#endif
