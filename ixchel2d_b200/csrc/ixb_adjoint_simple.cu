// ixb_adjoint_simple.cu -- discrete adjoint of the full coupled SIMPLE outer
// iteration (momentum, pressure correction, velocity/pressure update and
// energy, main.f90:404-1136 with one pass of each equation per outer
// iteration), for flows that depend on the temperature through buoyancy
// (natural and mixed convection).  The gradient is that of the hot-wall
// Nusselt number (ixb_nusselt_x, wall x = 0) after K outer iterations with
// respect to the Dirichlet value of every x-line on side a.  The reference
// has no counterpart.
//
// Every sweep of the iteration maps its input state s (the swept field and
// the fields its rows read) to x_out, where A(s) x_out = d(s) on the solved
// lines and x_out = x_in on the others.  Its adjoint, given lambda (the
// adjoint of x_out):
//   mu = A(s)^-T lambda                      (transposed batched line solve)
//   s_bar += sum over rows r of  mu_r d(d_r)/ds - mu_r (x_{r-1} d(a_r)/ds
//            + x_r d(b_r)/ds + x_{r+1} d(c_r)/ds)
//   x_in_bar += lambda                       (on the unsolved lines)
// The row's derivatives with respect to the ~10 stencil values it reads come
// from evaluating the row once more in forward-mode dual numbers, one
// derivative slot per stencil input, and the products with the weights
// (-mu x, mu) are scattered to the stencil positions with atomic adds.  The
// rows are restated here from ixb_device.cuh (the reference's formulas,
// mod_ec_momento.f90:365-1098, :145-355, mod_ec_energia.f90:119-443) in a
// form generic over the scalar type; the forward kernels are untouched.
// The velocity/pressure update (main.f90:931-962) has a hand-written adjoint.
//
// Forward: K outer iterations phase by phase (ixb_phase: the same kernels as
// the graph; the pressure loop starts from p' = 0), the state saved every C
// iterations.  Reverse, segment by segment from the last: restore the
// segment's checkpoint, recompute its iterations storing the state after
// every phase, then reverse the phases of each iteration from the last.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ixb_handle.h"
#include "ixb_nusselt.h"

namespace ixb {
namespace {

// ---------------------------------------------------------------------------
// forward-mode dual numbers with N derivative slots
// ---------------------------------------------------------------------------
template <int N>
struct Dual {
  double v;
  double d[N];
};

template <int N>
__device__ __forceinline__ Dual<N> cst(double x) {
  Dual<N> r;
  r.v = x;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = 0.0;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> seed(double x, int slot) {
  Dual<N> r = cst<N>(x);
  r.d[slot] = 1.0;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double s) {
  Dual<N> r;
  r.v = a.v * s;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * s;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(double s, const Dual<N>& a) { return a * s; }
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double s) {
  Dual<N> r = a;
  r.v += s;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  const double ib = 1.0 / b.v;
  r.v = a.v * ib;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double s) { return a * (1.0 / s); }
template <int N>
__device__ __forceinline__ Dual<N> operator/(double s, const Dual<N>& b) { return cst<N>(s) / b; }

// |x| and DMAX1(0, x) on plain doubles and on dual numbers
__device__ __forceinline__ double gabs(double x) { return fabs(x); }
template <int N>
__device__ __forceinline__ Dual<N> gabs(const Dual<N>& x) { return x.v < 0.0 ? -x : x; }
__device__ __forceinline__ double gpos(double x) { return x > 0.0 ? x : 0.0; }
template <int N>
__device__ __forceinline__ Dual<N> gpos(const Dual<N>& x) { return x.v > 0.0 ? x : cst<N>(0.0); }

// DMAX1(0, (1 - 0.1|P|)**5) and DMAX1(0, x)
template <class S>
__device__ __forceinline__ S aplaw(const S& pe) {
  const S t = 1.0 - 0.1 * gabs(pe);
  const S t2 = t * t;
  return gpos(t * (t2 * t2));
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(double s, const Dual<N>& a) {
  Dual<N> r = -a;
  r.v += s;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double s) {
  Dual<N> r = a;
  r.v -= s;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(double s, const Dual<N>& a) { return a + s; }

// ---------------------------------------------------------------------------
// the rows of the four equations, generic over the scalar type, from the
// stencil values x[0..12] (layouts in kStencil below).  Constants (metrics,
// mesh tables, u_ant / v_ant / T_ant, sources) are plain doubles.  The
// exact (IEEE-division) forms of ixb_device.cuh.
// ---------------------------------------------------------------------------
constexpr int NS = 13;  // stencil inputs of a row (the energy rows use 9)

template <class S>
struct GRow {
  S a, b, c, d;
};

// u momentum (ensambla_velu_x/_y, mod_ec_momento.f90:365-724) at (ii, jj)
template <class S>
__device__ GRow<S> row_u(const Geo<double>& G, const S* x, double u_ant, double fcon, double flin, int ii, int jj,
                         bool xform, S* aux) {
  const double fexu_i = G.met(M_FEXU, ii), fexu_m = G.met(M_FEXU, ii - 1), fexp_i = G.met(M_FEXP, ii);
  const S ud = fexu_i * x[1] + (1.0 - fexu_i) * x[0];
  const S ui = fexu_m * x[0] + (1.0 - fexu_m) * x[2];
  const S vn = fexp_i * x[6] + (1.0 - fexp_i) * x[5];
  const S vs = fexp_i * x[8] + (1.0 - fexp_i) * x[7];
  const S tint = fexp_i * x[10] + (1.0 - fexp_i) * x[9];
  const double g = G.gm, gamman = G.t(T_GU, ii, jj), gammas = G.t(T_GU, ii, jj - 1);
  const double di = G.met(M_DXP, ii), dd = G.met(M_DXP, ii + 1), ds = G.met(M_DYV, jj - 1), dn = G.met(M_DYV, jj);
  const double dx = G.met(M_DXU, ii), dy = G.met(M_DYU, jj);
  const S AI = -(G.t(T_CU1, ii, jj) * aplaw(ui * di / g) + gpos(ui * dy));
  const S AD = -(G.t(T_CU1, ii + 1, jj) * aplaw(ud * dd / g) + gpos(-ud * dy));
  const S BS = -(G.t(T_CU2, ii, jj - 1) * aplaw(vs * ds / gammas) + gpos(vs * dx));
  const S BN = -(G.t(T_CU2, ii, jj) * aplaw(vn * dn / gamman) + gpos(-vn * dx));
  const double dxdy = dx * dy;
  const S b = (-AI - AD - BS - BN - dxdy * flin + dxdy / G.dt) / G.rel_vel;
  const S rest = -dxdy * G.Ri * tint + dxdy * fcon + dxdy * u_ant / G.dt + (x[11] - x[12]) * dy +
                 b * (1.0 - G.rel_vel) * x[0];
  GRow<S> r;
  r.b = b;
  if (xform) { r.a = AI; r.c = AD; r.d = -BS * x[3] - BN * x[4] + rest; }
  else { r.a = BS; r.c = BN; r.d = -AI * x[2] - AD * x[1] + rest; }
  if (aux) *aux = b * G.rel_vel;
  return r;
}

// v momentum (ensambla_velv_x/_y, mod_ec_momento.f90:736-1098) at (ii, jj)
template <class S>
__device__ GRow<S> row_v(const Geo<double>& G, const S* x, double v_ant, double fcon, double flin, int ii, int jj,
                         bool xform, S* aux) {
  const double feyp_j = G.met(M_FEYP, jj), feyv_j = G.met(M_FEYV, jj), feyv_m = G.met(M_FEYV, jj - 1);
  const S ud = feyp_j * x[6] + (1.0 - feyp_j) * x[5];
  const S ui = feyp_j * x[8] + (1.0 - feyp_j) * x[7];
  const S vn = feyv_j * x[1] + (1.0 - feyv_j) * x[0];
  const S vs = feyv_m * x[0] + (1.0 - feyv_m) * x[2];
  const S tint = feyp_j * x[10] + (1.0 - feyp_j) * x[9];
  const double g = G.gm, gammad = G.t(T_GV, ii, jj), gammai = G.t(T_GV, ii - 1, jj);
  const double di = G.met(M_DXU, ii - 1), dd = G.met(M_DXU, ii), ds = G.met(M_DYP, jj), dn = G.met(M_DYP, jj + 1);
  const double dyv = G.met(M_DYV, jj), dxv = G.met(M_DXV, ii);
  const S AI = -(G.t(T_CV1, ii, jj) * aplaw(ui * di / gammai) + gpos(ui * dyv));
  const S AD = -(G.t(T_CV1, ii + 1, jj) * aplaw(ud * dd / gammad) + gpos(-ud * dyv));
  const S BS = -(G.t(T_CV2, ii, jj) * aplaw(vs * ds / g) + gpos(vs * dxv));
  const S BN = -(G.t(T_CV2, ii, jj + 1) * aplaw(vn * dn / g) + gpos(-vn * dxv));
  const double dxdy = dxv * dyv;
  const S b = (-AI - AD - BS - BN - dxdy * flin + dxdy / G.dt) / G.rel_vel;
  const S rest = -dxdy * G.Riy * tint + dxdy * fcon + dxdy * v_ant / G.dt + (x[11] - x[12]) * dxv +
                 b * (1.0 - G.rel_vel) * x[0];
  GRow<S> r;
  r.b = b;
  if (xform) { r.a = AI; r.c = AD; r.d = -BS * x[2] - BN * x[1] + rest; }
  else { r.a = BS; r.c = BN; r.d = -AI * x[3] - AD * x[4] + rest; }
  if (aux) *aux = b * G.rel_vel;
  return r;
}

// pressure correction (ensambla_corr_pres_x/_y, mod_ec_momento.f90:145-355) at (ii, jj)
template <class S>
__device__ GRow<S> row_p(const Geo<double>& G, const S* x, int ii, int jj, bool xform) {
  const double dyp = G.met(M_DYP, jj), dxp = G.met(M_DXP, ii);
  const S AI = -(dyp * dyp) / x[5], AD = -(dyp * dyp) / x[6];
  const S BS = -(dxp * dxp) / x[7], BN = -(dxp * dxp) / x[8];
  const S b = (-AI - AD - BS - BN) / G.rel_pres;
  const S bo = (x[10] - x[9]) * dyp + (x[12] - x[11]) * dxp;
  const S rest = bo + (1.0 - G.rel_pres) * b * x[0];
  GRow<S> r;
  r.b = b;
  if (xform) { r.a = AI; r.c = AD; r.d = -BS * x[3] - BN * x[4] + rest; }
  else { r.a = BS; r.c = BN; r.d = -AI * x[2] - AD * x[1] + rest; }
  return r;
}

// energy (ensambla_energia_x/_y, mod_ec_energia.f90:119-443) at (ii, jj)
template <class S>
__device__ GRow<S> row_t(const Geo<double>& G, const S* x, double T_ant, double fcon, double flin, int ii, int jj,
                         bool xform) {
  const S ud = x[5], ui = x[6], vn = x[7], vs = x[8];
  const double di = G.met(M_DXU, ii - 1), dd = G.met(M_DXU, ii), ds = G.met(M_DYV, jj - 1), dn = G.met(M_DYV, jj);
  const double dyp = G.met(M_DYP, jj), dxp = G.met(M_DXP, ii);
  const double gammad = G.met(M_HXU, ii), gammai = G.met(M_HXU, ii - 1);
  const double gamman = G.met(M_HYV, jj), gammas = G.met(M_HYV, jj - 1);
  const S AI = -(G.t(T_CT1, ii, jj) * aplaw(ui * di / gammai) + gpos(ui * dyp));
  const S AD = -(G.t(T_CT1, ii + 1, jj) * aplaw(ud * dd / gammad) + gpos(-ud * dyp));
  const S BS = -(G.t(T_CT2, ii, jj - 1) * aplaw(vs * ds / gammas) + gpos(vs * dxp));
  const S BN = -(G.t(T_CT2, ii, jj) * aplaw(vn * dn / gamman) + gpos(-vn * dxp));
  const double dxdy = dxp * dyp;
  const S b = (-AI - AD - BS - BN - dxdy * flin + dxdy / G.dt) / G.rel_ener;
  const S rest = dxdy * fcon + dxdy * T_ant / G.dt + b * (1.0 - G.rel_ener) * x[0];
  GRow<S> r;
  r.b = b;
  if (xform) { r.a = AI; r.c = AD; r.d = -BS * x[3] - BN * x[4] + rest; }
  else { r.a = BS; r.c = BN; r.d = -AI * x[2] - AD * x[1] + rest; }
  return r;
}

// ---------------------------------------------------------------------------
// stencils: the field and offset of every row input
// ---------------------------------------------------------------------------
enum Fld { F_U = 0, F_V, F_T, F_P, F_PC, F_AU, F_AV, F_COUNT, F_NONE = -1 };
struct Tap {
  int f, di, dj;
};
// groups: 0 u rows, 1 v rows, 2 p' rows, 3 T rows
__constant__ Tap kStencil[4][NS] = {
    {{F_U, 0, 0}, {F_U, 1, 0}, {F_U, -1, 0}, {F_U, 0, -1}, {F_U, 0, 1}, {F_V, 0, 0}, {F_V, 1, 0}, {F_V, 0, -1},
     {F_V, 1, -1}, {F_T, 0, 0}, {F_T, 1, 0}, {F_P, 0, 0}, {F_P, 1, 0}},
    {{F_V, 0, 0}, {F_V, 0, 1}, {F_V, 0, -1}, {F_V, -1, 0}, {F_V, 1, 0}, {F_U, 0, 0}, {F_U, 0, 1}, {F_U, -1, 0},
     {F_U, -1, 1}, {F_T, 0, 0}, {F_T, 0, 1}, {F_P, 0, 0}, {F_P, 0, 1}},
    {{F_PC, 0, 0}, {F_PC, 1, 0}, {F_PC, -1, 0}, {F_PC, 0, -1}, {F_PC, 0, 1}, {F_AU, -1, 0}, {F_AU, 0, 0},
     {F_AV, 0, -1}, {F_AV, 0, 0}, {F_U, 0, 0}, {F_U, -1, 0}, {F_V, 0, 0}, {F_V, 0, -1}},
    {{F_T, 0, 0}, {F_T, 1, 0}, {F_T, -1, 0}, {F_T, 0, -1}, {F_T, 0, 1}, {F_U, 0, 0}, {F_U, -1, 0}, {F_V, 0, 0},
     {F_V, 0, -1}, {F_NONE, 0, 0}, {F_NONE, 0, 0}, {F_NONE, 0, 0}, {F_NONE, 0, 0}}};

__host__ __device__ constexpr int eq_group(int eq) { return eq / 2 == 0 ? 0 : eq / 2 == 1 ? 1 : eq / 2 == 2 ? 2 : 3; }

// The pre-sweep state a sweep's rows read, its constants and boundary rows.
struct SweepState {
  const double* f[F_COUNT];   // u, v, T, p, p', au, av as the sweep reads them
  const double* x_out;        // the swept field after the sweep
  const double* ant;          // u_ant / v_ant / T_ant (null for p')
  const double* fcon;         // sources (null: none)
  const double* flin;
  const BCEntry* first;       // boundary rows (null: p', Dirichlet 0)
  const BCEntry* last;
  int eq, n, line_lo, line_hi;
};

template <class S>
__device__ __forceinline__ GRow<S> eval_row(const Geo<double>& G, const SweepState& s, const S* x, int ii, int jj,
                                            S* aux) {
  const bool X = (s.eq & 1) != 0;
  const int c0 = G.at(ii, jj);
  const double fc = s.fcon ? s.fcon[c0] : 0.0, fl = s.flin ? s.flin[c0] : 0.0;
  switch (eq_group(s.eq)) {
    case 0: return row_u(G, x, s.ant[c0], fc, fl, ii, jj, X, aux);
    case 1: return row_v(G, x, s.ant[c0], fc, fl, ii, jj, X, aux);
    case 2: return row_p(G, x, ii, jj, X);
    default: return row_t(G, x, s.ant[c0], fc, fl, ii, jj, X);
  }
}

__device__ __forceinline__ void cell_of(const SweepState& s, int L, int r, int& ii, int& jj) {
  if (s.eq & 1) { ii = r + 1; jj = L; }
  else { ii = L; jj = r + 1; }
}

// Forward rows (a, b, c) of every solved line at the pre-sweep state,
// contiguous per line: line L at (L - line_lo) * n.  Boundary rows follow
// impone_cond_frontera (p' rows: Dirichlet 0).
__global__ void adj_rows_kernel(const Geo<double> G, const SweepState s, double* __restrict__ fa,
                                double* __restrict__ fb, double* __restrict__ fc) {
  const int nl = s.line_hi - s.line_lo + 1;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nl * s.n) return;
  const int li = idx / s.n, r = idx - li * s.n, L = s.line_lo + li;
  double a, b, c;
  if (r == 0 || r == s.n - 1) {
    const BCEntry* t = r == 0 ? s.first : s.last;
    const int type = t ? t[L].type : 1;
    a = 0.0; b = 1.0; c = 0.0;
    if (type == 2) {
      if (r == 0) { b = -1.0; c = 1.0; }
      else { a = -1.0; }
    }
  } else {
    int ii, jj;
    cell_of(s, L, r, ii, jj);
    const int grp = eq_group(s.eq);
    double x[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const Tap tp = kStencil[grp][k];
      x[k] = tp.f == F_NONE ? 0.0 : s.f[tp.f][G.at(ii + tp.di, jj + tp.dj)];
    }
    const GRow<double> row = eval_row<double>(G, s, x, ii, jj, nullptr);
    a = row.a; b = row.b; c = row.c;
  }
  fa[idx] = a; fb[idx] = b; fc[idx] = c;
}

// Transposed rows (a'_r = c_{r-1}, b'_r = b_r, c'_r = a_{r+1}) with right-hand
// side lambda (the adjoint of the swept field after the sweep); the adjoint
// of the solved lines is then cleared (their x_in reaches x_out only through
// the rows, whose contributions adj_jac_kernel adds).
__global__ void adj_transpose_kernel(const Geo<double> G, const SweepState s, const double* __restrict__ fa,
                                     const double* __restrict__ fb, const double* __restrict__ fc,
                                     double* __restrict__ lam, double* __restrict__ ta, double* __restrict__ tb,
                                     double* __restrict__ tc, double* __restrict__ td) {
  const int nl = s.line_hi - s.line_lo + 1;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nl * s.n) return;
  const int li = idx / s.n, r = idx - li * s.n, L = s.line_lo + li;
  ta[idx] = r > 0 ? fc[idx - 1] : 0.0;
  tb[idx] = fb[idx];
  tc[idx] = r < s.n - 1 ? fa[idx + 1] : 0.0;
  int ii, jj;
  cell_of(s, L, r, ii, jj);
  const int c0 = G.at(ii, jj);
  td[idx] = lam[c0];
  lam[c0] = 0.0;
}

struct AdjFields {
  double* f[F_COUNT];  // adjoints of u, v, T, p, p', au, av (field layout)
};

// Contributions of every interior row of the solved lines to the adjoints of
// the stencil values it read: with mu_r from the transposed solve and x the
// swept field after the sweep, the weights of (a, b, c, d) are
// (-mu_r x_{r-1}, -mu_r x_r, -mu_r x_{r+1}, mu_r); aux_bar (u-x, v-x) adds
// au_bar * rel_vel to b's weight (au = b rel_vel).
__global__ void __launch_bounds__(128) adj_jac_kernel(const Geo<double> G, const SweepState s,
                                                      const double* __restrict__ mu, const double* aux_bar,
                                                      AdjFields adj) {
  const int nl = s.line_hi - s.line_lo + 1, rows = s.n - 2;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nl * rows) return;
  const int li = idx / rows, r = 1 + idx % rows, L = s.line_lo + li;
  int ii, jj, im, jm, ip, jp;
  cell_of(s, L, r, ii, jj);
  cell_of(s, L, r - 1, im, jm);
  cell_of(s, L, r + 1, ip, jp);
  const double m0 = mu[(size_t)li * s.n + r];
  const double wa = -m0 * s.x_out[G.at(im, jm)];
  double wb = -m0 * s.x_out[G.at(ii, jj)];
  const double wc = -m0 * s.x_out[G.at(ip, jp)];
  const double wd = m0;
  if (aux_bar) wb += aux_bar[G.at(ii, jj)] * G.rel_vel;
  if (wa == 0.0 && wb == 0.0 && wc == 0.0 && wd == 0.0) return;
  const int grp = eq_group(s.eq);
  Dual<NS> x[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    const Tap tp = kStencil[grp][k];
    x[k] = tp.f == F_NONE ? cst<NS>(0.0) : seed<NS>(s.f[tp.f][G.at(ii + tp.di, jj + tp.dj)], k);
  }
  const GRow<Dual<NS>> row = eval_row<Dual<NS>>(G, s, x, ii, jj, nullptr);
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    const Tap tp = kStencil[grp][k];
    if (tp.f == F_NONE) continue;
    const double g = wa * row.a.d[k] + wb * row.b.d[k] + wc * row.c.d[k] + wd * row.d.d[k];
    if (g != 0.0) atomicAdd(adj.f[tp.f] + G.at(ii + tp.di, jj + tp.dj), g);
  }
}

// Side-a boundary rows of the T x-sweep: row 0 of line jj is (0, 1, 0 | value)
// (or the Neumann row with the value as flux), so d x_out / d value = A^-1 e_0
// and the value's gradient is mu at row 0.
__global__ void adj_bcgrad_kernel(const SweepState s, const double* __restrict__ mu, double* __restrict__ grad) {
  const int li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li > s.line_hi - s.line_lo) return;
  grad[s.line_lo + li] += mu[(size_t)li * s.n];
}

// Adjoint of the velocity and pressure update (main.f90:931-962, correct_cell):
//   p += p_update p';  u(ii,jj) += dyu (p'(ii,jj) - p'(ii+1,jj)) / au;
//   v(ii,jj) += dxv (p'(ii,jj) - p'(ii,jj+1)) / av.
// u_bar, v_bar and p_bar pass through; p'_bar, au_bar and av_bar collect.
__global__ void adj_correct_kernel(const Geo<double> G, const double* __restrict__ pc, const double* __restrict__ au,
                                   const double* __restrict__ av, const double* __restrict__ ub,
                                   const double* __restrict__ vb, const double* __restrict__ pb, double* pcb,
                                   double* aub, double* avb) {
  const int ni = G.mi - 1;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ni * (G.nj - 1)) return;
  const int ii = 2 + idx % ni, jj = 2 + idx / ni;
  const int c0 = G.at(ii, jj);
  atomicAdd(pcb + c0, G.p_update * pb[c0]);
  if (ii <= G.mi - 1) {
    const double w = ub[c0];
    if (w != 0.0) {
      const int ce = G.at(ii + 1, jj);
      const double q = G.met(M_DYU, jj) / au[c0];
      atomicAdd(pcb + c0, w * q);
      atomicAdd(pcb + ce, -w * q);
      aub[c0] -= w * q * (pc[c0] - pc[ce]) / au[c0];
    }
  }
  if (jj <= G.nj - 1) {
    const double w = vb[c0];
    if (w != 0.0) {
      const int cn = G.at(ii, jj + 1);
      const double q = G.met(M_DXV, ii) / av[c0];
      atomicAdd(pcb + c0, w * q);
      atomicAdd(pcb + cn, -w * q);
      avb[c0] -= w * q * (pc[c0] - pc[cn]) / av[c0];
    }
  }
}

}  // namespace
}  // namespace ixb

using namespace ixb;

#define SCK(x)                   \
  do {                           \
    cudaError_t e_ = (x);        \
    if (e_ != cudaSuccess) {     \
      h->last_cuda = e_;         \
      return IXB_ECUDA;          \
    }                            \
  } while (0)
#define STRY(x)                  \
  do {                           \
    const int s_ = (x);          \
    if (s_ != IXB_OK) return s_; \
  } while (0)

namespace {

// the fields stored after every phase of one outer iteration
enum Snap { S_U0 = 0, S_V0, S_P0, S_T0, S_U1, S_U2, S_AU, S_V1, S_V2, S_AV, S_PC1, S_PC2, S_U3, S_V3, S_T1, S_T2,
            S_COUNT };

struct SimpleAdjoint {
  ixb_handle* h;
  size_t fsz = 0;
  Geo<double> G{};
  std::vector<void*> allocs;
  double* store = nullptr;  // C iterations x S_COUNT fields
  double* ckpt = nullptr;   // (segments + 1) x (u, v, p, T)
  AdjFields adj{};
  double *fa = nullptr, *fb = nullptr, *fc = nullptr, *ta = nullptr, *tb = nullptr, *tc = nullptr, *td = nullptr,
         *mu = nullptr, *gd = nullptr;

  ~SimpleAdjoint() {
    if (h && h->stream) cudaStreamSynchronize(h->stream);
    for (void* p : allocs) cudaFree(p);
  }
  int alloc(double** p, size_t n) {
    if (cudaMalloc((void**)p, n * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return IXB_ENOMEM;
    }
    allocs.push_back(*p);
    return IXB_OK;
  }

  int init(int C, int segments) {
    fsz = h->fsz;
    G = handle_geo(h);
    STRY(alloc(&store, (size_t)C * S_COUNT * fsz));
    STRY(alloc(&ckpt, (size_t)(segments + 1) * 4 * fsz));
    for (int k = 0; k < F_COUNT; ++k) {
      STRY(alloc(&adj.f[k], fsz));
      SCK(cudaMemsetAsync(adj.f[k], 0, fsz * sizeof(double), h->stream));
    }
    const size_t nst = (size_t)std::max(h->mi + 1, h->nj + 1) * (size_t)std::max(h->mi + 1, h->nj + 1);
    for (double** p : {&fa, &fb, &fc, &ta, &tb, &tc, &td, &mu}) STRY(alloc(p, nst));
    STRY(alloc(&gd, (size_t)h->nj + 2));
    SCK(cudaMemsetAsync(gd, 0, ((size_t)h->nj + 2) * sizeof(double), h->stream));
    return IXB_OK;
  }

  int copy(double* dst, const double* src) {
    SCK(cudaMemcpyAsync(dst, src, fsz * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    return IXB_OK;
  }
  int save(double* dst) {
    STRY(copy(dst, h->u[h->cu]));
    STRY(copy(dst + fsz, h->v[h->cv]));
    STRY(copy(dst + 2 * fsz, h->p));
    return copy(dst + 3 * fsz, h->T[h->cT]);
  }
  int restore(const double* src) {
    STRY(copy(h->u[h->cu], src));
    STRY(copy(h->v[h->cv], src + fsz));
    STRY(copy(h->p, src + 2 * fsz));
    return copy(h->T[h->cT], src + 3 * fsz);
  }

  // One outer iteration, one pass of each equation, phase by phase; with
  // `st`, the state after every phase is stored there.
  int iterate(double* st) {
    auto snap = [&](int k, const double* src) { return st ? copy(st + (size_t)k * fsz, src) : IXB_OK; };
    STRY(snap(S_U0, h->u[h->cu]));
    STRY(snap(S_V0, h->v[h->cv]));
    STRY(snap(S_P0, h->p));
    STRY(snap(S_T0, h->T[h->cT]));
    STRY(ixb_phase(h, 0));
    STRY(snap(S_U1, h->u[h->cu]));
    STRY(ixb_phase(h, 1));
    STRY(snap(S_U2, h->u[h->cu]));
    STRY(snap(S_AU, h->au));
    STRY(ixb_phase(h, 2));
    STRY(snap(S_V1, h->v[h->cv]));
    STRY(ixb_phase(h, 3));
    STRY(snap(S_V2, h->v[h->cv]));
    STRY(snap(S_AV, h->av));
    SCK(cudaMemsetAsync(h->pc[h->cpc], 0, fsz * sizeof(double), h->stream));  // p' starts from zero
    STRY(ixb_phase(h, 4));
    STRY(snap(S_PC1, h->pc[h->cpc]));
    STRY(ixb_phase(h, 5));
    STRY(snap(S_PC2, h->pc[h->cpc]));
    STRY(ixb_phase(h, 6));
    STRY(snap(S_U3, h->u[h->cu]));
    STRY(snap(S_V3, h->v[h->cv]));
    STRY(ixb_phase(h, 7));
    STRY(snap(S_T1, h->T[h->cT]));
    STRY(ixb_phase(h, 8));
    return snap(S_T2, h->T[h->cT]);
  }

  // the boundary tables of variable var (0 u, 1 v, 2 T) for x- or y-lines
  void tables(SweepState& s, int var) {
    const bool x = (s.eq & 1) != 0;
    const BCEntry* base = h->bc + (size_t)var * 4 * h->bcstride;
    s.first = base + (size_t)(x ? 0 : 1) * h->bcstride;
    s.last = base + (size_t)(x ? 2 : 3) * h->bcstride;
  }
  SweepState state(int eq, const double* st) {
    SweepState s{};
    s.eq = eq;
    const SweepShape sh = sweep_shape(eq, h->mi, h->nj, 8, 1, 128);
    s.n = sh.n;
    s.line_lo = sh.line_lo;
    s.line_hi = sh.line_hi;
    auto S = [&](int k) { return st + (size_t)k * fsz; };
    switch (eq) {
      case EQ_UY: case EQ_UX:
        s.f[F_U] = S(eq == EQ_UY ? S_U0 : S_U1); s.f[F_V] = S(S_V0); s.f[F_T] = S(S_T0); s.f[F_P] = S(S_P0);
        s.x_out = S(eq == EQ_UY ? S_U1 : S_U2); s.ant = h->u_ant; s.fcon = h->fcon[0]; s.flin = h->flin[0];
        tables(s, 0);
        break;
      case EQ_VY: case EQ_VX:
        s.f[F_V] = S(eq == EQ_VY ? S_V0 : S_V1); s.f[F_U] = S(S_U2); s.f[F_T] = S(S_T0); s.f[F_P] = S(S_P0);
        s.x_out = S(eq == EQ_VY ? S_V1 : S_V2); s.ant = h->v_ant; s.fcon = h->fcon[1]; s.flin = h->flin[1];
        tables(s, 1);
        break;
      case EQ_PY: case EQ_PX:
        s.f[F_PC] = eq == EQ_PY ? h->zero : S(S_PC1); s.f[F_AU] = S(S_AU); s.f[F_AV] = S(S_AV);
        s.f[F_U] = S(S_U2); s.f[F_V] = S(S_V2);
        s.x_out = S(eq == EQ_PY ? S_PC1 : S_PC2);
        break;
      default:
        s.f[F_T] = S(eq == EQ_TY ? S_T0 : S_T1); s.f[F_U] = S(S_U3); s.f[F_V] = S(S_V3);
        s.x_out = S(eq == EQ_TY ? S_T1 : S_T2); s.ant = h->T_ant; s.fcon = h->fcon[2]; s.flin = h->flin[2];
        tables(s, 2);
        break;
    }
    return s;
  }

  // One sweep reversed: lam (the swept field's adjoint) holds the adjoint of
  // x_out on entry and of x_in on exit; the other fields' adjoints collect.
  int sweep_back(const SweepState& s, double* lam, const double* aux_bar, bool bc_grad) {
    const int nl = s.line_hi - s.line_lo + 1, rows = nl * s.n;
    adj_rows_kernel<<<(rows + 255) / 256, 256, 0, h->stream>>>(G, s, fa, fb, fc);
    SCK(cudaGetLastError());
    adj_transpose_kernel<<<(rows + 255) / 256, 256, 0, h->stream>>>(G, s, fa, fb, fc, lam, ta, tb, tc, td);
    SCK(cudaGetLastError());
    SCK(tridiag_f64(ta, tb, tc, td, mu, s.n, nl, 0, IXB_SOLVER_HYBRID, h->stream));
    if (bc_grad) {
      adj_bcgrad_kernel<<<(nl + 127) / 128, 128, 0, h->stream>>>(s, mu, gd);
      SCK(cudaGetLastError());
    }
    const int cells = nl * (s.n - 2);
    adj_jac_kernel<<<(cells + 127) / 128, 128, 0, h->stream>>>(G, s, mu, aux_bar, adj);
    SCK(cudaGetLastError());
    return IXB_OK;
  }

  // One outer iteration reversed, from its stored phases.
  int iteration_back(const double* st) {
    auto S = [&](int k) { return st + (size_t)k * fsz; };
    STRY(sweep_back(state(EQ_TX, st), adj.f[F_T], nullptr, true));
    STRY(sweep_back(state(EQ_TY, st), adj.f[F_T], nullptr, false));
    const int ncell = (h->mi - 1) * (h->nj - 1);
    adj_correct_kernel<<<(ncell + 255) / 256, 256, 0, h->stream>>>(G, S(S_PC2), S(S_AU), S(S_AV), adj.f[F_U],
                                                                 adj.f[F_V], adj.f[F_P], adj.f[F_PC], adj.f[F_AU],
                                                                 adj.f[F_AV]);
    SCK(cudaGetLastError());
    STRY(sweep_back(state(EQ_PX, st), adj.f[F_PC], nullptr, false));
    STRY(sweep_back(state(EQ_PY, st), adj.f[F_PC], nullptr, false));
    SCK(cudaMemsetAsync(adj.f[F_PC], 0, fsz * sizeof(double), h->stream));  // p' starts from the zero field
    STRY(sweep_back(state(EQ_VX, st), adj.f[F_V], adj.f[F_AV], false));
    SCK(cudaMemsetAsync(adj.f[F_AV], 0, fsz * sizeof(double), h->stream));  // av is written by the v-x sweep
    STRY(sweep_back(state(EQ_VY, st), adj.f[F_V], nullptr, false));
    STRY(sweep_back(state(EQ_UX, st), adj.f[F_U], adj.f[F_AU], false));
    SCK(cudaMemsetAsync(adj.f[F_AU], 0, fsz * sizeof(double), h->stream));  // au is written by the u-x sweep
    return sweep_back(state(EQ_UY, st), adj.f[F_U], nullptr, false);
  }

  // lambda_T = d Nu / d T: the Nusselt number is linear in T; its weights
  // are evaluated on unit fields with the shared host/device formula
  int objective(int j0, int j1) {
    const int mi = h->mi, nj = h->nj;
    std::vector<double> along(nj + 2, 0.0), across(mi + 2, 0.0);
    for (int j = 1; j <= nj + 1; ++j) along[j] = h->yp[j - 1];
    for (int i = 1; i <= mi + 1; ++i) across[i] = h->xp[i - 1];
    std::vector<double> w(fsz, 0.0);
    for (int k = j0; k <= j1 + 2; ++k)
      for (int l = 1; l <= 3; ++l) {
        auto f = [&](int kk, int ll) { return (kk == k && ll == l) ? 1.0 : 0.0; };
        w[(size_t)(k - 1) * h->LD + (l - 1)] = nusselt_wall(f, along.data(), across.data(), mi + 1, 0, 0, j0, j1);
      }
    SCK(cudaMemcpyAsync(adj.f[F_T], w.data(), fsz * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    SCK(cudaStreamSynchronize(h->stream));
    return IXB_OK;
  }
};

}  // namespace

extern "C" int ixb_adjoint_simple(ixb_handle* h, int K, int C, int j0, int j1, double* grad, double* nu0) {
  if (!h || K < 1 || C < 1) return IXB_EINVAL;
  STRY(handle_ready(h));
  if (h->prec != IXB_PREC_FP64) return IXB_EINVAL;  // the refined form's line solves are another map
  if (j0 < 1 || j1 < j0) return IXB_EINVAL;
  for (int k = j0; k <= j1; k += 2)
    if (k + 2 > h->nj + 1) return IXB_EINVAL;
  const int segments = (K + C - 1) / C;
  SimpleAdjoint A{h};
  STRY(A.init(std::min(C, K), segments));
  // forward, with a checkpoint at the start of every segment and at the end
  for (int sgm = 0; sgm < segments; ++sgm) {
    STRY(A.save(A.ckpt + (size_t)sgm * 4 * A.fsz));
    const int count = std::min(C, K - sgm * C);
    for (int it = 0; it < count; ++it) STRY(A.iterate(nullptr));
  }
  STRY(A.save(A.ckpt + (size_t)segments * 4 * A.fsz));
  double nu = 0.0;
  STRY(ixb_nusselt_x(h, j0, j1, &nu, nullptr));
  if (nu0) *nu0 = nu;
  if (!grad) return IXB_OK;
  STRY(A.objective(j0, j1));
  for (int sgm = segments - 1; sgm >= 0; --sgm) {
    STRY(A.restore(A.ckpt + (size_t)sgm * 4 * A.fsz));
    const int count = std::min(C, K - sgm * C);
    for (int it = 0; it < count; ++it) STRY(A.iterate(A.store + (size_t)it * S_COUNT * A.fsz));
    for (int it = count - 1; it >= 0; --it) STRY(A.iteration_back(A.store + (size_t)it * S_COUNT * A.fsz));
  }
  STRY(A.restore(A.ckpt + (size_t)segments * 4 * A.fsz));  // the state of the forward run
  std::vector<double> g((size_t)h->nj + 2);
  SCK(cudaMemcpyAsync(g.data(), A.gd, g.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  SCK(cudaStreamSynchronize(h->stream));
  int timed_out = 0;
  SCK(tridiag_take_timeout(&timed_out));
  if (timed_out) return IXB_ETIMEOUT;
  for (int jj = 1; jj <= h->nj + 1; ++jj) grad[jj - 1] = g[jj];
  return IXB_OK;
}
