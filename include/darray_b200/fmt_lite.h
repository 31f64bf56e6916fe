// The part of the {fmt} library's API that DArray's tests and headers call -- fmt::format and fmt::print with
// "{}" placeholders (no format specifications) -- written here from that API's documented behaviour, so code
// written against the reference's headers (which include the vendored fmt) compiles against this mirror.  Each
// "{}" takes the next argument as std::ostream << prints it; "{{" and "}}" print braces.
#pragma once
#include <cstdio>
#include <sstream>
#include <string>
#include <utility>

namespace fmt {
namespace lite_detail {
inline void emit(std::ostringstream& os, const char*& f) {
  for (; *f; ++f) {
    if ((f[0] == '{' && f[1] == '{') || (f[0] == '}' && f[1] == '}')) {
      os << *f;
      ++f;
    } else {
      os << *f;
    }
  }
}
template <typename A, typename... Rest>
void emit(std::ostringstream& os, const char*& f, A&& a, Rest&&... rest) {
  for (; *f; ++f) {
    if ((f[0] == '{' && f[1] == '{') || (f[0] == '}' && f[1] == '}')) {
      os << *f;
      ++f;
    } else if (f[0] == '{') {
      while (*f && *f != '}') ++f;  // "{...}": the next argument, whatever the specification
      if (*f) ++f;
      os << a;
      emit(os, f, std::forward<Rest>(rest)...);
      return;
    } else {
      os << *f;
    }
  }
}
}  // namespace lite_detail

template <typename... Args>
std::string format(const std::string& fmt_str, Args&&... args) {
  std::ostringstream os;
  const char* f = fmt_str.c_str();
  lite_detail::emit(os, f, std::forward<Args>(args)...);
  return os.str();
}

template <typename... Args>
void print(const std::string& fmt_str, Args&&... args) {
  const std::string s = format(fmt_str, std::forward<Args>(args)...);
  std::fwrite(s.data(), 1, s.size(), stdout);
}
}  // namespace fmt
