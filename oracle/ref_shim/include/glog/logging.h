/*
 * glog/logging.h — the logging and CHECK macros the reference's engine path
 * uses, for the oracle shim (test infrastructure only).
 *
 * Each LOG / PLOG / LOG_IF statement builds its text in a stream and, at the
 * end of the statement, hands (severity, text) to plato_shim_log_sink when the
 * shim has set one (the shim reads the reference's per-epoch lines from
 * there), else drops it.  A failed CHECK prints its text and aborts, as glog
 * does; FATAL aborts after its line.
 */
#ifndef PLATO_ORACLE_SHIM_GLOG_H
#define PLATO_ORACLE_SHIM_GLOG_H

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>

namespace google {
enum LogSeverity { GLOG_INFO = 0, GLOG_WARNING = 1, GLOG_ERROR = 2, GLOG_FATAL = 3 };
inline void InitGoogleLogging(const char*) {}
inline void ShutdownGoogleLogging() {}
inline void InstallFailureSignalHandler() {}
}  // namespace google

typedef void (*plato_shim_log_sink_t)(int severity, const char* text);
inline plato_shim_log_sink_t& plato_shim_log_sink() {
  static plato_shim_log_sink_t sink = nullptr;
  return sink;
}

namespace plato_shim_glog {

class message {
 public:
  message(int severity, bool fatal, bool with_errno = false)
      : severity_(severity), fatal_(fatal), errno_(with_errno ? errno : 0) {}
  ~message() {
    if (errno_) os_ << ": " << std::strerror(errno_) << " [" << errno_ << "]";
    const std::string s = os_.str();
    if (plato_shim_log_sink()) plato_shim_log_sink()(severity_, s.c_str());
    if (fatal_) {
      std::fprintf(stderr, "F %s\n", s.c_str());
      std::abort();
    }
  }
  std::ostream& stream() { return os_; }

 private:
  int severity_;
  bool fatal_;
  int errno_;
  std::ostringstream os_;
};

/* turns `stream << ...` into void, so the macros below can sit in ?: */
struct voidify {
  void operator&(std::ostream&) {}
};

}  // namespace plato_shim_glog

#define PLATO_SHIM_SEV_INFO 0
#define PLATO_SHIM_SEV_WARNING 1
#define PLATO_SHIM_SEV_ERROR 2
#define PLATO_SHIM_SEV_FATAL 3

#define LOG(sev) plato_shim_glog::message(PLATO_SHIM_SEV_##sev, PLATO_SHIM_SEV_##sev == 3).stream()
#define PLOG(sev) plato_shim_glog::message(PLATO_SHIM_SEV_##sev, PLATO_SHIM_SEV_##sev == 3, true).stream()
#define LOG_IF(sev, cond) \
  !(cond) ? (void)0 : plato_shim_glog::voidify() & LOG(sev)
#define VLOG(n) LOG_IF(INFO, false)
#define DLOG(sev) LOG_IF(sev, false)

#define CHECK(cond)                                                                  \
  (cond) ? (void)0                                                                   \
         : plato_shim_glog::voidify() &                                              \
               plato_shim_glog::message(3, true).stream() << "Check failed: " #cond " "
#define PLATO_SHIM_CHECK_OP(a, b, op) CHECK((a)op(b))
#define CHECK_EQ(a, b) PLATO_SHIM_CHECK_OP(a, b, ==)
#define CHECK_NE(a, b) PLATO_SHIM_CHECK_OP(a, b, !=)
#define CHECK_LT(a, b) PLATO_SHIM_CHECK_OP(a, b, <)
#define CHECK_LE(a, b) PLATO_SHIM_CHECK_OP(a, b, <=)
#define CHECK_GT(a, b) PLATO_SHIM_CHECK_OP(a, b, >)
#define CHECK_GE(a, b) PLATO_SHIM_CHECK_OP(a, b, >=)
#define CHECK_NOTNULL(p) (p)
#define DCHECK(cond) CHECK(true || (cond))
#define DCHECK_EQ(a, b) DCHECK((a) == (b))
#define DCHECK_NE(a, b) DCHECK((a) != (b))
#define DCHECK_LT(a, b) DCHECK((a) < (b))
#define DCHECK_LE(a, b) DCHECK((a) <= (b))
#define DCHECK_GT(a, b) DCHECK((a) > (b))
#define DCHECK_GE(a, b) DCHECK((a) >= (b))

#endif
