// ixb_listdir.h -- Fortran list-directed record reader and Dw.d output for
// the reference's text files (host only).
#pragma once
#include <cstdio>
#include <string>
#include <vector>

namespace ixb {

class ListReader {
 public:
  explicit ListReader(const char* path);
  ~ListReader();
  bool ok() const { return f_ != nullptr; }
  // One READ statement: `count` items from the next record(s); the rest of
  // the last record is discarded.  Returns false at end of file.
  bool read(std::vector<std::string>& items, int count);

 private:
  bool next_line(std::string& line);
  FILE* f_ = nullptr;
};

bool parse_real(const std::string& t, double* out);
bool parse_int(const std::string& t, int* out);
bool parse_logical(const std::string& t, int* out);
std::string fortran_char(const std::string& t, size_t len);
int bc_type_code(const std::string& tipo4);
// x as Fortran D23.15 writes it (right-justified in 23 columns)
std::string fmt_d23_15(double x);

}  // namespace ixb
