// ixb_host.cpp -- host-side inputs of the hot path that need no GPU:
// boundary-table construction (lectura_cond_frontera,
// source/mod_cond_frontera.f90:70-245) and the boundary-condition file reader.
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ixb.h"
#include "ixb_listdir.h"

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
