// ixb_nusselt.h -- the wall-averaged Nusselt number of nusselt_promedio_y
// (source/mod_postproceso.f90:100-215) and its vertical-wall counterpart, as
// one host/device function: the device kernel evaluates it on the field, the
// adjoint evaluates it on unit fields to get its (linear) weights.
#pragma once
#include <cuda_runtime.h>

namespace ixb {

// The three terms panel ii (ii = k0, k0+2, ...) adds to the integral of
// dT/dn along the wall: the quadratic through the wall derivative at ii,
// ii+1, ii+2 integrated over [x_ii, x_ii+2].  f(k, l): temperature at
// position k along the wall and l across it (l = 1 at the wall of index 1);
// along/across: 1-based node coordinates.  wall 0: the wall at index 1,
// wall 1: the one at n_across.  With `quirk` set (the reference rule) the
// wall derivative is known only on k0..k1 and reads as 0 beyond, as derivada
// does in the reference.
template <class F>
__host__ __device__ void nusselt_panel(F f, const double* along, const double* across, int n_across, int wall,
                                       int quirk, int k1, int ii, double* t3) {
  const int jj = wall == 0 ? 1 : n_across - 2;
  double der[3];
  for (int q = 0; q < 3; ++q) {
    const int k = ii + q;
    if (quirk && k > k1) { der[q] = 0.0; continue; }  // derivada beyond i_1o stays 0
    const double dy1 = f(k, jj + 1) - f(k, jj), dy2 = f(k, jj + 2) - f(k, jj + 1);
    const double dx1 = across[jj + 1] - across[jj], dx2 = across[jj + 2] - across[jj + 1];
    const double a = (dy2 / dx2 - dy1 / dx1) / (dx1 + dx2);
    const double b = dy2 / dx2 - a * (across[jj + 1] + across[jj + 2]);
    der[q] = 2.0 * a * (wall == 0 ? across[jj] : across[jj + 2]) + b;
  }
  const double x_o = along[ii], x_1 = along[ii + 1], x_2 = along[ii + 2];
  const double y_o = der[0], y_1 = der[1], y_2 = der[2];
  const double alpha = ((y_2 - y_1) / (x_2 - x_1) - (y_1 - y_o) / (x_1 - x_o)) / (x_2 - x_o);
  const double beta = (y_2 - y_1) / (x_2 - x_1) - alpha * (x_1 + x_2);
  const double gamma = y_o - alpha * x_o * x_o - beta * x_o;
  t3[0] = alpha / 3.0 * (x_2 * x_2 * x_2 - x_o * x_o * x_o);
  t3[1] = beta / 2.0 * (x_2 * x_2 - x_o * x_o);
  t3[2] = gamma * (x_2 - x_o);
}

// -(integral of dT/dn along the wall) over panels k0..k1 (step 2), summed in
// panel order as nu = nu + t0 + t1 + t2 (left to right), the reference's
// accumulation.
template <class F>
__host__ __device__ double nusselt_wall(F f, const double* along, const double* across, int n_across, int wall,
                                        int quirk, int k0, int k1) {
  double nu = 0.0;
  for (int ii = k0; ii <= k1; ii += 2) {
    double t[3];
    nusselt_panel(f, along, across, n_across, wall, quirk, k1, ii, t);
    nu = nu + t[0] + t[1] + t[2];
  }
  return -nu;
}

}  // namespace ixb
