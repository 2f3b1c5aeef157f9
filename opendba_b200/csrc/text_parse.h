// Text values: the input format's line parser and the output writers'
// number formatter.
//
// Line values of the text input format (one value per line, the first
// whitespace-separated token; cpu_utils.hpp:92-134 reads each with
// std::stringstream >> T).  parse_line_value gives the same value as that
// extraction in the "C" locale, faster: a plain decimal token
//   [+-] digits [. digits] [(e|E) [+-] digits]   (at least one mantissa digit)
// is what the stream's parser accumulates for a float, and it converts the
// accumulated text with strtof / strtod (correctly rounded), so such a token
// is converted here directly with std::from_chars (also correctly rounded);
// every other line (no digits, inf / nan text, hex, an exponent without
// digits, a result out of range) goes through the stream itself.
#pragma once

#include <cctype>
#include <charconv>
#include <cmath>
#include <sstream>
#include <string>
#include <system_error>

namespace odba {

inline bool text_space(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}
inline bool text_digit(char c) { return c >= '0' && c <= '9'; }

// The value of the line [b, e), as std::stringstream(line) >> v gives it
// (v = 0 when the extraction fails).
template <typename T>
T parse_line_value(const char *b, const char *e) {
  const char *p = b;
  while (p < e && text_space(*p)) ++p;
  const char *q = p;
  if (q < e && (*q == '+' || *q == '-')) ++q;
  int mant = 0;
  while (q < e && text_digit(*q)) ++q, ++mant;
  if (q < e && *q == '.') {
    ++q;
    while (q < e && text_digit(*q)) ++q, ++mant;
  }
  bool plain = mant > 0;
  if (plain && q < e && (*q == 'e' || *q == 'E')) {
    const char *x = q + 1;
    if (x < e && (*x == '+' || *x == '-')) ++x;
    int ed = 0;
    while (x < e && text_digit(*x)) ++x, ++ed;
    if (ed > 0)
      q = x;
    else
      plain = false;  // the stream's parser treats a bare exponent mark differently
  }
  // a token followed directly by a letter or another mark may extend the
  // stream's grammar (hex, inf/nan); leave those to the stream
  if (plain && q < e && (std::isalpha(static_cast<unsigned char>(*q)) || *q == '.'))
    plain = false;
  if (plain) {
    // from_chars takes no leading '+'; the value is the same without it
    const char *s = *p == '+' ? p + 1 : p;
    T v = T(0);
    const std::from_chars_result r = std::from_chars(s, q, v, std::chars_format::general);
    if (r.ec == std::errc() && r.ptr == q && std::isfinite(v)) return v;
  }
  std::stringstream in(std::string(b, e));
  T v = T(0);
  in >> v;
  return v;
}

// Appends v as `std::ostream << v` prints it with the default flags and
// precision (6): the stream formats through printf's %.6g, and std::to_chars
// in the general format with precision 6 is specified to give the same
// characters ("as if by printf"; a float is formatted from its exact value,
// as the stream's promotion to double keeps it).  Infinities and NaNs go
// through the stream itself.  Three to four times faster than the stream.
template <typename T>
inline void append_stream_value(std::string &out, T v) {
  if (std::isfinite(v)) {
    char buf[48];
    const std::to_chars_result r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::general, 6);
    if (r.ec == std::errc()) {
      out.append(buf, r.ptr);
      return;
    }
  }
  std::ostringstream s;
  s << v;
  out += s.str();
}

}  // namespace odba
