// Minimal logging used by the drop-in headers: spdlog::info / warn / error
// with "{}" placeholders. info is printed only when PM_LOG is set in the
// environment; warn and error always go to stderr.
#pragma once
#include <cstdlib>
#include <iostream>
#include <sstream>

namespace spdlog {
namespace pm_detail {
inline void put(std::ostringstream& os, const char* f) { os << f; }
template <class T, class... R>
void put(std::ostringstream& os, const char* f, const T& v, const R&... r) {
  for (; *f; ++f) {
    if (f[0] == '{' && f[1] == '}') {
      os << v;
      put(os, f + 2, r...);
      return;
    }
    os << *f;
  }
}
template <class... A>
void log(const char* level, const char* f, const A&... a) {
  std::ostringstream os;
  put(os, f, a...);
  std::cerr << "[" << level << "] " << os.str() << '\n';
}
}  // namespace pm_detail
template <class... A>
void info(const char* f, const A&... a) {
  if (std::getenv("PM_LOG")) pm_detail::log("info", f, a...);
}
template <class... A>
void warn(const char* f, const A&... a) {
  pm_detail::log("warning", f, a...);
}
template <class... A>
void error(const char* f, const A&... a) {
  pm_detail::log("error", f, a...);
}
}  // namespace spdlog
