// ixb_listdir.cpp -- Fortran list-directed input and D23.15 output for the
// reference's text files (host only).  Compiled into libixb.so and into the
// ixchel2d_gpu driver.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ixb.h"
#include "ixb_listdir.h"

namespace ixb {

// ---------------------------------------------------------------------------
// Fortran list-directed input: every READ starts at a new record, takes as
// many values as it needs (continuing onto further records), and discards
// the rest of its last record -- which is why trailing "! comment" text in
// the reference's .dat files is harmless.
// ---------------------------------------------------------------------------
ListReader::ListReader(const char* path) { f_ = std::fopen(path, "r"); }
ListReader::~ListReader() { if (f_) std::fclose(f_); }

bool ListReader::next_line(std::string& line) {
  line.clear();
  if (!f_) return false;
  int ch;
  bool any = false;
  while ((ch = std::fgetc(f_)) != EOF) {
    any = true;
    if (ch == '\n') break;
    if (ch != '\r') line.push_back((char)ch);
  }
  return any;
}

static void split_tokens(const std::string& s, std::vector<std::string>& out) {
  size_t i = 0;
  const size_t n = s.size();
  while (i < n) {
    while (i < n && (std::isspace((unsigned char)s[i]) || s[i] == ',')) ++i;
    if (i >= n) break;
    if (s[i] == '/') break;  // slash ends the input list
    if (s[i] == '\'' || s[i] == '"') {
      const char q = s[i++];
      std::string tok;
      while (i < n) {
        if (s[i] == q) {
          if (i + 1 < n && s[i + 1] == q) { tok.push_back(q); i += 2; continue; }
          ++i;
          break;
        }
        tok.push_back(s[i++]);
      }
      out.push_back(tok);
      continue;
    }
    size_t j = i;
    while (j < n && !std::isspace((unsigned char)s[j]) && s[j] != ',' && s[j] != '/') ++j;
    out.push_back(s.substr(i, j - i));
    i = j;
  }
}

bool ListReader::read(std::vector<std::string>& items, int count) {
  items.clear();
  std::string line;
  while ((int)items.size() < count) {
    if (!next_line(line)) return false;
    std::vector<std::string> toks;
    split_tokens(line, toks);
    for (auto& t : toks) {
      if ((int)items.size() >= count) break;
      items.push_back(t);
    }
  }
  return true;
}

// A Fortran real: D or E exponents, and the exponent-letter-free form that
// Dw.d / Ew.d output takes for |exponent| > 99 ("0.25-120").
bool parse_real(const std::string& t, double* out) {
  std::string s = t;
  for (auto& ch : s)
    if (ch == 'd' || ch == 'D') ch = 'e';
  if (s.empty()) return false;
  if (s.find_first_of("eE") == std::string::npos) {
    const size_t k = s.find_first_of("+-", 1);
    if (k != std::string::npos && (std::isdigit((unsigned char)s[k - 1]) || s[k - 1] == '.')) s.insert(k, 1, 'e');
  }
  char* end = nullptr;
  const double v = std::strtod(s.c_str(), &end);
  if (end == s.c_str() || *end != '\0') return false;
  *out = v;
  return true;
}

bool parse_int(const std::string& t, int* out) {
  if (t.empty()) return false;
  char* end = nullptr;
  const long v = std::strtol(t.c_str(), &end, 10);
  if (end == t.c_str() || *end != '\0') return false;
  *out = (int)v;
  return true;
}

bool parse_logical(const std::string& t, int* out) {
  std::string s = t;
  size_t k = 0;
  if (!s.empty() && s[0] == '.') k = 1;
  if (k >= s.size()) return false;
  const char c = (char)std::toupper((unsigned char)s[k]);
  if (c == 'T') { *out = 1; return true; }
  if (c == 'F') { *out = 0; return true; }
  return false;
}

// character(len=L) assignment of a list-directed token: truncate or pad
std::string fortran_char(const std::string& t, size_t len) {
  std::string s = t.substr(0, std::min(len, t.size()));
  return s;
}

int bc_type_code(const std::string& tipo4) {
  if (tipo4 == "diri") return IXB_BC_DIRI;
  if (tipo4 == "neum") return IXB_BC_NEUM;
  return IXB_BC_OTHER;
}

// Fortran Dw.d output of x with w = 23, d = 15: "0.ddddddddddddddd" mantissa,
// exponent "D+ee" (|e| <= 99) or "+eee" (the D dropped for |e| > 99),
// right-justified.  The 15 digits are those of the correctly rounded
// %.14E conversion.
std::string fmt_d23_15(double x) {
  char buf[64];
  std::string mant, exps;
  if (x == 0.0 || !std::isfinite(x)) {
    if (!std::isfinite(x)) {
      std::snprintf(buf, sizeof buf, "%23s", std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity"));
      return buf;
    }
    mant = "0.000000000000000";
    exps = "D+00";
  } else {
    std::snprintf(buf, sizeof buf, "%.14E", std::fabs(x));  // d.ddddddddddddddE+xx
    const char* e = std::strchr(buf, 'E');
    const int ex = std::atoi(e + 1) + 1;
    std::string digits;
    digits.push_back(buf[0]);
    digits.append(buf + 2, (size_t)(e - (buf + 2)));
    mant = "0." + digits;
    const int ax = ex < 0 ? -ex : ex;
    char eb[16];
    if (ax <= 99) std::snprintf(eb, sizeof eb, "D%c%02d", ex < 0 ? '-' : '+', ax);
    else std::snprintf(eb, sizeof eb, "%c%03d", ex < 0 ? '-' : '+', ax);
    exps = eb;
  }
  std::string s = (x < 0 ? "-" : "") + mant + exps;
  if (s.size() < 23) s.insert(0, 23 - s.size(), ' ');
  return s;
}

}  // namespace ixb
