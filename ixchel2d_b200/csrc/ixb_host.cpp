// ixb_host.cpp -- host-side inputs of the hot path that need no GPU:
// boundary-table construction (lectura_cond_frontera,
// source/mod_cond_frontera.f90:70-245) and the Fortran list-directed record
// reader used to parse the reference's input files.
#include <cctype>
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

}  // namespace ixb

using namespace ixb;

extern "C" {

// lectura_cond_frontera index rule, source/mod_cond_frontera.f90:125-149
// (side a; b, c, d are the same with their own coordinate and size):
// indice_div(1) = 2; for each division, indice_div(k+1) = the first grid
// index whose coordinate exceeds x1 (size+1 if none); finally
// indice_div(ndivis+1) = size-1.  x0 is read but not used by the reference.
int ixb_bc_locate(int side, int ndivis, const double* x1, const int* type, const double* value, const double* xx,
                  int mm, const double* yy, int nn, ixb_bc_side* out) {
  if (!out || side < 0 || side > 3 || ndivis < 0 || ndivis > 15) return IXB_EINVAL;
  if (ndivis > 0 && (!x1 || !type || !value)) return IXB_EINVAL;
  const bool on_y = (side == 0 || side == 2);
  const double* coord = on_y ? yy : xx;
  const int size = on_y ? nn : mm;
  if (!coord || size < 2) return IXB_EINVAL;
  std::memset(out, 0, sizeof(*out));
  out->side = side;
  out->ndivis = ndivis;
  out->index[0] = 2;
  for (int k = 0; k < ndivis; ++k) {
    out->type[k] = type[k];
    out->value[k] = value[k];
    int kk = 1;
    for (; kk <= size; ++kk)
      if (coord[kk - 1] > x1[k]) break;
    out->index[k + 1] = kk;
  }
  out->index[ndivis] = size - 1;
  return IXB_OK;
}

// lectura_cond_frontera file reader, source/mod_cond_frontera.f90:109-240.
// xx (mm entries) / yy (nn entries) are the coordinates of the variable's
// nodes along x / y.  Sides absent from the file keep ndivis = 0.
int ixb_read_bc_file(const char* path, const double* xx, int mm, const double* yy, int nn, ixb_bc_side out[4]) {
  if (!path || !out) return IXB_EINVAL;
  ListReader rd(path);
  if (!rd.ok()) return IXB_EIO;
  for (int s = 0; s < 4; ++s) {
    std::memset(&out[s], 0, sizeof(out[s]));
    out[s].side = s;
  }
  std::vector<std::string> it;
  for (int rec = 0; rec < 4; ++rec) {
    if (!rd.read(it, 3)) return IXB_EIO;
    const std::string lado = fortran_char(it[1], 1);
    int ndiv = 0;
    if (!parse_int(it[2], &ndiv) || ndiv < 0 || ndiv > 15) return IXB_EIO;
    double x1[15];
    int type[15];
    double val[15];
    for (int k = 0; k < ndiv; ++k) {
      if (!rd.read(it, 4)) return IXB_EIO;
      double x0;
      if (!parse_real(it[0], &x0) || !parse_real(it[1], &x1[k]) || !parse_real(it[3], &val[k])) return IXB_EIO;
      type[k] = bc_type_code(fortran_char(it[2], 4));
    }
    int side = -1;
    if (lado == "a") side = 0;
    else if (lado == "b") side = 1;
    else if (lado == "c") side = 2;
    else if (lado == "d") side = 3;
    if (side < 0) continue;  // select case matches no side: record consumed, nothing stored
    const int st = ixb_bc_locate(side, ndiv, x1, type, val, xx, mm, yy, nn, &out[side]);
    if (st != IXB_OK) return st;
  }
  return IXB_OK;
}

}  // extern "C"
