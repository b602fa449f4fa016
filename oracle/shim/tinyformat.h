// Minimal stand-in for tinyformat's tfm::format, used only to compile the
// reference sources into the CPU oracle (oracle/_ref).  The reference pins
// tinyformat at commit 3a33bbf65442432277eee079e83d3e8fac51730c
// (third_party/deps.bzl:16-23); that library is not vendored, so this header
// restates the one entry point the reference uses: printf-style formatting of
// arbitrary streamable arguments.
//
// Supported: flags [-+ 0#], width, .precision, length modifiers (ignored),
// conversions d i u x X o c s g G f F e E p and %%.  Integer conversions cast
// the argument to a 64-bit integer; anything else is streamed with <<.
#pragma once

#include <cstdint>
#include <cstdio>
#include <ostream>
#include <sstream>
#include <string>
#include <type_traits>

namespace tfm {
namespace detail {

struct spec_t {
  std::string flags;
  int width = -1, precision = -1;
  char conv = 's';
};

// Parse one conversion starting just after '%'.  Returns the index after it.
inline size_t parse_spec(const char* fmt, size_t i, spec_t& s) {
  while (fmt[i] && std::string("-+ 0#").find(fmt[i]) != std::string::npos)
    s.flags.push_back(fmt[i++]);
  if (fmt[i] >= '0' && fmt[i] <= '9') {
    s.width = 0;
    while (fmt[i] >= '0' && fmt[i] <= '9') s.width = 10 * s.width + (fmt[i++] - '0');
  }
  if (fmt[i] == '.') {
    i++;
    s.precision = 0;
    while (fmt[i] >= '0' && fmt[i] <= '9') s.precision = 10 * s.precision + (fmt[i++] - '0');
  }
  while (fmt[i] == 'l' || fmt[i] == 'h' || fmt[i] == 'z' || fmt[i] == 'j' || fmt[i] == 't' ||
         fmt[i] == 'L' || fmt[i] == 'q')
    i++;
  if (fmt[i]) s.conv = fmt[i++];
  return i;
}

inline std::string printf_spec(const spec_t& s, const char* length, char conv) {
  std::string f = "%" + s.flags;
  if (s.width >= 0) f += std::to_string(s.width);
  if (s.precision >= 0) f += "." + std::to_string(s.precision);
  f += length;
  f.push_back(conv);
  return f;
}

inline void pad(std::ostream& out, const std::string& body, const spec_t& s) {
  const bool left = s.flags.find('-') != std::string::npos;
  const int fill = s.width > int(body.size()) ? s.width - int(body.size()) : 0;
  if (!left) out << std::string(fill, ' ');
  out << body;
  if (left) out << std::string(fill, ' ');
}

template<class T> void format_one(std::ostream& out, const spec_t& s, const T& value) {
  using D = std::decay_t<T>;
  char buf[128];
  if constexpr (std::is_integral_v<D> || std::is_enum_v<D>) {
    const char c = s.conv;
    if (c == 'd' || c == 'i') {
      snprintf(buf, sizeof(buf), printf_spec(s, "ll", 'd').c_str(), (long long)value);
      out << buf;
      return;
    } else if (c == 'u' || c == 'x' || c == 'X' || c == 'o') {
      snprintf(buf, sizeof(buf), printf_spec(s, "ll", c).c_str(),
               (unsigned long long)(std::make_unsigned_t<std::conditional_t<std::is_enum_v<D>, int, D>>)value);
      out << buf;
      return;
    } else if (c == 'c') {
      pad(out, std::string(1, char(value)), s);
      return;
    } else if (c == 'g' || c == 'G' || c == 'f' || c == 'F' || c == 'e' || c == 'E') {
      snprintf(buf, sizeof(buf), printf_spec(s, "", c).c_str(), double(value));
      out << buf;
      return;
    }
    if constexpr (std::is_same_v<D, char>) {
      pad(out, std::string(1, value), s);
    } else {
      std::ostringstream o;
      o << +value;
      pad(out, o.str(), s);
    }
    return;
  } else if constexpr (std::is_floating_point_v<D>) {
    const char c = (s.conv == 's' || s.conv == 'd') ? 'g' : s.conv;
    snprintf(buf, sizeof(buf), printf_spec(s, "", c).c_str(), double(value));
    out << buf;
    return;
  } else if constexpr (std::is_pointer_v<D> && !std::is_same_v<D, const char*> &&
                       !std::is_same_v<D, char*>) {
    snprintf(buf, sizeof(buf), "%p", (const void*)value);
    pad(out, buf, s);
    return;
  } else {
    std::ostringstream o;
    if (s.precision >= 0) o.precision(s.precision);
    o << value;
    std::string body = o.str();
    if (s.conv == 's' && s.precision >= 0 && int(body.size()) > s.precision &&
        (std::is_same_v<D, const char*> || std::is_same_v<D, char*> || std::is_same_v<D, std::string>))
      body.resize(s.precision);
    pad(out, body, s);
  }
}

inline void format_rest(std::ostream& out, const char* fmt, size_t i) {
  for (; fmt[i]; i++) {
    if (fmt[i] == '%' && fmt[i + 1] == '%') { out << '%'; i++; }
    else out << fmt[i];
  }
}

template<class T, class... Rest>
void format_rest(std::ostream& out, const char* fmt, size_t i, const T& first, const Rest&... rest) {
  for (; fmt[i]; i++) {
    if (fmt[i] != '%') { out << fmt[i]; continue; }
    if (fmt[i + 1] == '%') { out << '%'; i++; continue; }
    spec_t s;
    const size_t next = parse_spec(fmt, i + 1, s);
    format_one(out, s, first);
    format_rest(out, fmt, next, rest...);
    return;
  }
}

}  // namespace detail

template<class... Args> void format(std::ostream& out, const char* fmt, const Args&... args) {
  detail::format_rest(out, fmt, 0, args...);
}

template<class... Args> std::string format(const char* fmt, const Args&... args) {
  std::ostringstream out;
  detail::format_rest(out, fmt, 0, args...);
  return out.str();
}

template<class... Args> std::string format(const std::string& fmt, const Args&... args) {
  return format(fmt.c_str(), args...);
}

template<class... Args> void format(std::ostream& out, const std::string& fmt, const Args&... args) {
  format(out, fmt.c_str(), args...);
}

}  // namespace tfm
