// ixb_files.cpp -- mesh generation and the mesh/state files of Ixchel2D
// (host only, no GPU).
//
// * ixb_mesh_axis / ixb_staggered_mesh: the u/v node distributions of
//   malla/malla_irr.f90 (unif :97-100, tubo :81-89, cent :54-64) plus a
//   two-sided tanh wall clustering the reference lacks, and the p nodes at the
//   midpoints with one extrapolated node half a cell outside each wall
//   (:66-77, :101-106).  Coordinates are rounded to the 15 significant digits
//   of the D23.15 files, so a generated mesh equals what the reference reads
//   back from its own files.
// * ixb_write_state_files / ixb_read_state_files: the three files of a mesh
//   and state (malla_irr.f90:176-203 writes them, mod_malla.f90:137-162 reads
//   them): a list-directed header "i_0 i_1 iter a", then one record per node
//   in the order DO jj / DO ii: "x y u" (3D23.15) for u, "x y v" for v and
//   "x y T p" (4D23.15) for the p/T nodes.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ixb.h"
#include "ixb_listdir.h"

namespace {

double round_d23_15(double x) {
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.14E", x);
  return std::strtod(buf, nullptr);
}

}  // namespace

using ixb::fmt_d23_15;

extern "C" {

int ixb_mesh_axis(int kind, int n, double length, double param, double centre, double* nodes) {
  if (n < 2 || !nodes) return IXB_EINVAL;
  for (int i = 0; i < n; ++i) {
    const double s = (double)i / (double)(n - 1);  // malla_irr.f90:49-51
    double x;
    switch (kind) {
      case IXB_MESH_UNIF:
        x = length * 1.0 * s;
        break;
      case IXB_MESH_TUBO: {  // erf clustering at both walls, ky = 10, my = 0.8
        const double ky = 10.0, my = 0.8;
        x = length * 1.0 * (0.5 + my * (s - 0.5) + 0.5 * (1 - my) * std::erf(ky * (s - 0.5)) / std::erf(0.5 * ky));
        break;
      }
      case IXB_MESH_CENT: {  // sinh clustering around `centre`, tau = param
        const double tau = param;
        const double b = 1.0 / (2.0 * tau) *
                         std::log((1.0 + (std::exp(tau) - 1.0) * (centre / length)) /
                                  (1.0 + (std::exp(-tau) - 1.0) * (centre / length)));
        x = centre * (1.0 + std::sinh(tau * (s - b)) / std::sinh(tau * b));
        break;
      }
      case IXB_MESH_TANH:  // two-sided tanh wall clustering (no counterpart in malla_irr.f90)
        x = length * (1.0 + std::tanh(param * (2.0 * s - 1.0)) / std::tanh(param)) / 2.0;
        break;
      default:
        return IXB_EINVAL;
    }
    nodes[i] = x;
  }
  return IXB_OK;
}

int ixb_staggered_mesh(int mi, int nj, int xkind, double xparam, int ykind, double yparam, double ao, double bo,
                       double* xu, double* yv, double* xp, double* yp) {
  if (mi < 3 || nj < 3 || !xu || !yv || !xp || !yp) return IXB_EINVAL;
  int st = ixb_mesh_axis(xkind, mi, ao, xparam, 0.5 * ao, xu);
  if (st != IXB_OK) return st;
  st = ixb_mesh_axis(ykind, nj, bo, yparam, 0.5 * bo, yv);
  if (st != IXB_OK) return st;
  auto pnodes = [](const double* f, int n, double* p) {
    p[0] = (3.0 * f[0] - f[1]) / 2.0;
    for (int i = 0; i < n - 1; ++i) p[i + 1] = (f[i + 1] + f[i]) / 2.0;
    p[n] = (3.0 * f[n - 1] - f[n - 2]) / 2.0;
  };
  pnodes(xu, mi, xp);
  pnodes(yv, nj, yp);
  for (int i = 0; i < mi; ++i) xu[i] = round_d23_15(xu[i]);
  for (int j = 0; j < nj; ++j) yv[j] = round_d23_15(yv[j]);
  for (int i = 0; i <= mi; ++i) xp[i] = round_d23_15(xp[i]);
  for (int j = 0; j <= nj; ++j) yp[j] = round_d23_15(yp[j]);
  return IXB_OK;
}

int ixb_write_state_files(const char* ufile, const char* vfile, const char* pfile, int mi, int nj, const double* xu,
                          const double* yv, const double* xp, const double* yp, const double* u, const double* v,
                          const double* T, const double* p, int i0, int i1, int iter, double a) {
  if (!ufile || !vfile || !pfile || mi < 2 || nj < 2 || !xu || !yv || !xp || !yp || !u || !v || !T || !p)
    return IXB_EINVAL;
  auto write = [&](const char* path, int nx, int ny, const double* xs, const double* ys, const double* f,
                   const double* g) -> bool {
    FILE* fp = std::fopen(path, "w");
    if (!fp) return false;
    std::fprintf(fp, " %11d %11d %11d %s\n", i0, i1, iter, fmt_d23_15(a).c_str());
    std::string line;
    for (int jj = 0; jj < ny; ++jj)
      for (int ii = 0; ii < nx; ++ii) {
        const size_t k = (size_t)jj * nx + ii;  // Fortran (ii, jj), column-major
        line = fmt_d23_15(xs[ii]) + fmt_d23_15(ys[jj]) + fmt_d23_15(f[k]);
        if (g) line += fmt_d23_15(g[k]);
        line.push_back('\n');
        if (std::fputs(line.c_str(), fp) < 0) { std::fclose(fp); return false; }
      }
    return std::fclose(fp) == 0;
  };
  if (!write(ufile, mi, nj + 1, xu, yp, u, nullptr)) return IXB_EIO;
  if (!write(vfile, mi + 1, nj, xp, yv, v, nullptr)) return IXB_EIO;
  if (!write(pfile, mi + 1, nj + 1, xp, yp, T, p)) return IXB_EIO;
  return IXB_OK;
}

int ixb_read_state_files(const char* ufile, const char* vfile, const char* pfile, int mi, int nj, double* xu,
                         double* yv, double* xp, double* yp, double* u, double* v, double* T, double* p, int* i0,
                         int* i1, int* iter, double* a) {
  if (!ufile || !vfile || !pfile || mi < 2 || nj < 2 || !xu || !yv || !xp || !yp || !u || !v || !T || !p)
    return IXB_EINVAL;
  auto read = [&](const char* path, int nx, int ny, double* xs, double* ys, double* f, double* g) -> int {
    ixb::ListReader rd(path);
    if (!rd.ok()) return IXB_EIO;
    std::vector<std::string> it;
    if (!rd.read(it, 4)) return IXB_EIO;
    int h0 = 0, h1 = 0, hi = 0;
    double ha = 0.0;
    if (!ixb::parse_int(it[0], &h0) || !ixb::parse_int(it[1], &h1) || !ixb::parse_int(it[2], &hi) ||
        !ixb::parse_real(it[3], &ha))
      return IXB_EIO;
    if (i0) *i0 = h0;
    if (i1) *i1 = h1;
    if (iter) *iter = hi;
    if (a) *a = ha;
    const int per = g ? 4 : 3;
    for (int jj = 0; jj < ny; ++jj)
      for (int ii = 0; ii < nx; ++ii) {
        if (!rd.read(it, per)) return IXB_EIO;
        const size_t k = (size_t)jj * nx + ii;
        double x, y;
        if (!ixb::parse_real(it[0], &x) || !ixb::parse_real(it[1], &y) || !ixb::parse_real(it[2], f + k))
          return IXB_EIO;
        if (g && !ixb::parse_real(it[3], g + k)) return IXB_EIO;
        xs[ii] = x;  // the last record of each coordinate wins, as in the reference's loop
        ys[jj] = y;
      }
    return IXB_OK;
  };
  int st = read(ufile, mi, nj + 1, xu, yp, u, nullptr);
  if (st != IXB_OK) return st;
  st = read(vfile, mi + 1, nj, xp, yv, v, nullptr);
  if (st != IXB_OK) return st;
  return read(pfile, mi + 1, nj + 1, xp, yp, T, p);
}

}  // extern "C"
