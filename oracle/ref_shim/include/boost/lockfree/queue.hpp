/* boost/lockfree/queue.hpp — for the oracle shim (test infrastructure only):
 * a mutex-guarded queue with the members the reference calls. */
#ifndef PLATO_ORACLE_SHIM_BOOST_LOCKFREE_QUEUE_HPP
#define PLATO_ORACLE_SHIM_BOOST_LOCKFREE_QUEUE_HPP
#include <cstddef>
#include <deque>
#include <mutex>
namespace boost {
namespace lockfree {
template <typename T>
class queue {
 public:
  explicit queue(std::size_t = 0) {}
  bool push(const T& v) {
    std::lock_guard<std::mutex> lock(mu_);
    q_.push_back(v);
    return true;
  }
  bool pop(T& v) {
    std::lock_guard<std::mutex> lock(mu_);
    if (q_.empty()) return false;
    v = q_.front();
    q_.pop_front();
    return true;
  }
  bool empty() {
    std::lock_guard<std::mutex> lock(mu_);
    return q_.empty();
  }
  bool is_lock_free() const { return true; }

 private:
  std::mutex mu_;
  std::deque<T> q_;
};
}  // namespace lockfree
}  // namespace boost
#endif
