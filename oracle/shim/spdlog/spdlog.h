// ORACLE shim — test infrastructure only. A project-written stand-in for the
// spdlog calls the reference headers make (spdlog::info/warn/error with
// "{}" placeholders), so that the reference compiles without the spdlog
// library. info is silent unless PM_REF_LOG is set; warn/error go to stderr.
#pragma once
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>

namespace spdlog {
namespace detail {
inline void fmt_into(std::ostringstream& os, const char* f) { os << f; }
template <class T, class... R>
void fmt_into(std::ostringstream& os, const char* f, const T& v, const R&... r) {
  for (; *f; ++f) {
    if (f[0] == '{' && f[1] == '}') {
      os << v;
      fmt_into(os, f + 2, r...);
      return;
    }
    os << *f;
  }
}
template <class... A>
void emit(const char* level, const char* f, const A&... a) {
  std::ostringstream os;
  fmt_into(os, f, a...);
  std::cerr << "[" << level << "] " << os.str() << "\n";
}
}  // namespace detail
template <class... A>
void info(const char* f, const A&... a) {
  if (std::getenv("PM_REF_LOG")) detail::emit("info", f, a...);
}
template <class... A>
void warn(const char* f, const A&... a) {
  detail::emit("warn", f, a...);
}
template <class... A>
void error(const char* f, const A&... a) {
  detail::emit("error", f, a...);
}
}  // namespace spdlog
