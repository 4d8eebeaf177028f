// Minimal stand-in for glog's LOG() used when the reference's GPU solvers are
// compiled into oracle/_ref (test infrastructure): LOG(INFO) lines go to
// stdout prefixed with "I ", LOG(FATAL) aborts.
#pragma once
#include <cstdlib>
#include <iostream>
#include <sstream>

namespace google {
struct LogLine {
  std::ostringstream s;
  bool fatal;
  explicit LogLine(bool f) : fatal(f) {}
  ~LogLine() {
    std::cout << (fatal ? "F " : "I ") << s.str() << std::endl;
    if (fatal) std::abort();
  }
  template <typename T>
  LogLine &operator<<(const T &v) {
    s << v;
    return *this;
  }
};
}  // namespace google
#define GPM_SHIM_LOG_INFO false
#define GPM_SHIM_LOG_WARNING false
#define GPM_SHIM_LOG_ERROR false
#define GPM_SHIM_LOG_FATAL true
#define LOG(sev) google::LogLine(GPM_SHIM_LOG_##sev)
