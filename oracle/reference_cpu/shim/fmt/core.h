// TEST INFRASTRUCTURE ONLY.
//
// A minimal stand-in for the {fmt} calls in the reference's modules:
// fmt::print and fmt::format with "{}" / "{:spec}" / "{n:spec}" fields,
// where each argument is written with iostream's default formatting (the
// format spec is not interpreted; these strings are messages and file
// names, not data).
#pragma once

#include <cstdio>
#include <sstream>
#include <string>
#include <string_view>
#include <vector>

namespace fmt {
namespace detail {

template <class T>
std::string to_s(const T &x) {
  std::ostringstream os;
  os << x;
  return os.str();
}

inline std::string substitute(std::string_view f, const std::vector<std::string> &args) {
  std::string out;
  size_t next = 0;
  for (size_t i = 0; i < f.size(); ++i) {
    const char ch = f[i];
    if (ch == '{' && i + 1 < f.size() && f[i + 1] == '{') {
      out += '{';
      ++i;
    } else if (ch == '}' && i + 1 < f.size() && f[i + 1] == '}') {
      out += '}';
      ++i;
    } else if (ch == '{') {
      const size_t close = f.find('}', i);
      if (close == std::string_view::npos) break;
      std::string_view field = f.substr(i + 1, close - i - 1);
      const size_t colon = field.find(':');
      std::string_view index = field.substr(0, colon);
      size_t a = next++;
      if (!index.empty()) a = (size_t)std::stoul(std::string(index));
      if (a < args.size()) out += args[a];
      i = close;
    } else {
      out += ch;
    }
  }
  return out;
}

}  // namespace detail

template <class... A>
std::string format(std::string_view f, const A &...a) {
  return detail::substitute(f, {detail::to_s(a)...});
}

template <class... A>
void print(std::string_view f, const A &...a) {
  const std::string s = format(f, a...);
  std::fwrite(s.data(), 1, s.size(), stdout);
}

}  // namespace fmt
