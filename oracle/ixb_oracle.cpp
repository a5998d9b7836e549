// ixb_oracle.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// CPU restatement of Ixchel2D's SIMPLE outer iteration (the reference is
// Fortran 90 + OpenACC).  It is the checker for the CUDA path and the timed
// CPU baseline: only tests/, __graft_entry__.smoke() and bench.py's CPU legs
// load it.  The product library never links or calls it.
//
// Parity status: UNPINNED against outputs of the reference itself.  The
// reference is Fortran and no Fortran compiler (gfortran, nvfortran, flang,
// ifx) exists in this image, and the reference ships no golden vectors, tests
// or fixtures.  This restatement is instead pinned by known-answer tests
// (tests/test_oracle.py): Thomas vs dense LU, pure-diffusion coefficients,
// conduction-only cavity -> linear profile and Nu = 1, mirror symmetry,
// vanishing u-residual at convergence.
//
// Arithmetic: IEEE binary64, evaluated left to right exactly as the Fortran
// statements are written, built with -ffp-contract=off (no FMA contraction).
// `x**5` is restated as x*((x*x)*(x*x)) (binary powering, what gfortran's
// __builtin_powi expands to).
//
// Every routine cites the reference statement(s) it restates
// (source/<file>:<line>).  Arrays keep the Fortran shapes, column-major,
// 1-based, including the shared coefficient scratch AI/AC/AD/Rx (mi+1,nj+1)
// and BS/BC/BN/Ry (nj+1,mi+1) of source/main.f90:114-115.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct A2 {  // Fortran array real(DBL) :: x(n1, n2), 1-based
  int n1 = 0, n2 = 0;
  std::vector<double> d;
  void init(int a, int b, double v = 0.0) { n1 = a; n2 = b; d.assign((size_t)a * b, v); }
  inline double& operator()(int i, int j) { return d[(size_t)(j - 1) * n1 + (i - 1)]; }
  inline double* col(int j) { return &d[(size_t)(j - 1) * n1]; }
  void fill(double v) { std::fill(d.begin(), d.end(), v); }
};

// tipo_cond_front, source/mod_cond_frontera.f90:25-38 (indice_div widened to
// 16 entries so that 15 divisions fit; the reference declares 14).
struct BCSide {
  char lado = 'z';
  int ndivis = 0;
  int tipo[15] = {0};      // 1 = 'diri', 2 = 'neum', 0 = anything else ('desc')
  double valor[15] = {0};
  int indice[16] = {0};    // indice_div(1..ndivis+1)
  // Extension (no counterpart in the reference, whose sides hold at most 15
  // piecewise-constant segments): when set, the value written on line l is
  // line_val[l-1] instead of its segment's valor -- the per-line boundary
  // values of the GPU library's ixb_set_bc_values.
  std::vector<double> line_val;
};

// x**5 with the reference's integer power: DMAX1(0, (1-0.1|P|)**5)
// (e.g. source/mod_ec_momento.f90:513).
static inline double plaw(double pe) {
  double t = 1.0 - 0.1 * std::fabs(pe);
  double t2 = t * t;
  double t5 = t * (t2 * t2);
  return std::fmax(0.0, t5);
}
static inline double dmax0(double x) { return std::fmax(0.0, x); }

struct Case {
  int mi = 0, nj = 0;
  // mesh, source/mod_malla.f90:39-52 (1-based, index 0 unused)
  std::vector<double> xu, yv, xp, yp, deltaxp, deltayp, deltaxu, deltayu, deltaxv, deltayv,
      fexp, feyp, fexu, feyv;
  // parameters, source/main.f90:164-244
  double dt = 1.0, rel_vel = 0.7, rel_pres = 0.3, rel_ener = 0.9;
  double conv_u = 1e30, conv_p = 1e30, conv_t = 1e30, conv_resi = 0, conv_paso = 0;
  double p_update = 0.6;  // hard-coded 0.6 of source/main.f90:934
  int iter_ecuaci_max = 0, iter_simple_max = 0;
  int iter_ecuaci = 0, iter_simple = 0;
  double maxbo = 0, residuo = 0, err_u = 0, err_p = 0, err_t = 0;
  int64_t n_momen = 0, n_pres = 0, n_ener = 0, n_simple = 0;
  // fields, source/mod_ec_momento.f90:27-41 and mod_ec_energia.f90:23-30
  A2 u, u_ant, au, Resu, fu, Ri, fcon_u, flin_u;      // (mi, nj+1)
  A2 v, v_ant, av, fv, fcon_v, flin_v;                // (mi+1, nj)
  A2 pres, corr_pres, fcorr_pres, b_o, gamma_momen, Riy;  // (mi+1, nj+1)
  A2 temp, temp_ant, ftemp, gamma_energ, fcon_t, flin_t;  // (mi+1, nj+1)
  A2 AI, AC, AD, Rx;  // (mi+1, nj+1)
  A2 BS, BC, BN, Ry;  // (nj+1, mi+1)
  BCSide bcu[4], bcv[4], bct[4];

  void alloc(int mi_, int nj_) {
    mi = mi_; nj = nj_;
    auto v1 = [](std::vector<double>& x, int n) { x.assign(n + 1, 0.0); };
    v1(xu, mi); v1(yv, nj); v1(xp, mi + 1); v1(yp, nj + 1);
    v1(deltaxp, mi); v1(deltayp, nj); v1(deltaxu, mi); v1(deltayu, nj);
    v1(deltaxv, mi); v1(deltayv, nj); v1(fexp, mi); v1(feyp, nj); v1(fexu, mi); v1(feyv, nj);
    for (A2* a : {&u, &u_ant, &au, &Resu, &fu, &Ri, &fcon_u, &flin_u}) a->init(mi, nj + 1);
    for (A2* a : {&v, &v_ant, &av, &fv, &fcon_v, &flin_v}) a->init(mi + 1, nj);
    for (A2* a : {&pres, &corr_pres, &fcorr_pres, &b_o, &gamma_momen, &Riy, &temp, &temp_ant,
                  &ftemp, &gamma_energ, &fcon_t, &flin_t, &AI, &AC, &AD, &Rx})
      a->init(mi + 1, nj + 1);
    for (A2* a : {&BS, &BC, &BN, &Ry}) a->init(nj + 1, mi + 1);
    au.fill(1.e40);  // source/main.f90:309-310
    av.fill(1.e40);
  }

  // lectura_mallas_escalonadas metric part, source/mod_malla.f90:167-218
  void metrics() {
    for (int ii = 2; ii <= mi; ++ii) deltaxp[ii] = xu[ii] - xu[ii - 1];
    for (int jj = 2; jj <= nj; ++jj) deltayp[jj] = yv[jj] - yv[jj - 1];
    for (int ii = 1; ii <= mi; ++ii) deltaxu[ii] = xp[ii + 1] - xp[ii];
    for (int jj = 2; jj <= nj; ++jj) deltayu[jj] = yv[jj] - yv[jj - 1];
    for (int ii = 2; ii <= mi; ++ii) deltaxv[ii] = xu[ii] - xu[ii - 1];
    for (int jj = 1; jj <= nj; ++jj) deltayv[jj] = yp[jj + 1] - yp[jj];
    for (int ii = 1; ii <= mi; ++ii) fexp[ii] = (xp[ii + 1] - xu[ii]) / (xp[ii + 1] - xp[ii]);
    for (int jj = 1; jj <= nj; ++jj) feyp[jj] = (yp[jj + 1] - yv[jj]) / (yp[jj + 1] - yp[jj]);
    for (int ii = 1; ii <= mi - 1; ++ii)
      fexu[ii] = (xu[ii + 1] - xp[ii + 1]) / (xu[ii + 1] - xu[ii]);
    for (int jj = 1; jj <= nj - 1; ++jj)
      feyv[jj] = (yv[jj + 1] - yp[jj + 1]) / (yv[jj + 1] - yv[jj]);
  }

  // ---------------------------------------------------------------------
  // Assembly routines.  Argument binding follows the CALL sites in main.f90
  // (which matters for ensambla_energia_*: main passes fexu/feyv into the
  // dummies named fexpo/feypo, source/main.f90:990 and :1061).
  // ---------------------------------------------------------------------

  // ensambla_velu_x, source/mod_ec_momento.f90:365-541, called at main.f90:499
  void velu_x(int ii, int jj) {
    A2& g = gamma_momen;
    double ud = fexu[ii] * u(ii + 1, jj) + (1.0 - fexu[ii]) * u(ii, jj);
    double ui = fexu[ii - 1] * u(ii, jj) + (1.0 - fexu[ii - 1]) * u(ii - 1, jj);
    double vn = fexp[ii] * v(ii + 1, jj) + (1.0 - fexp[ii]) * v(ii, jj);
    double vs = fexp[ii] * v(ii + 1, jj - 1) + (1.0 - fexp[ii]) * v(ii, jj - 1);
    double gammad = (g(ii + 1, jj + 1) * g(ii + 1, jj)) /
                    (g(ii + 1, jj + 1) * (1.0 - feyp[jj]) + g(ii + 1, jj) * feyp[jj]);
    double gammai = (g(ii, jj + 1) * g(ii, jj)) /
                    (g(ii, jj + 1) * (1.0 - feyp[jj]) + g(ii, jj) * feyp[jj]);
    double gamman = gammai * gammad / (gammad * (1.0 - fexp[ii]) + gammai * fexp[ii]);
    gammad = (g(ii + 1, jj) * g(ii + 1, jj - 1)) /
             (g(ii + 1, jj) * (1.0 - feyp[jj - 1]) + g(ii + 1, jj - 1) * feyp[jj - 1]);
    gammai = (g(ii, jj) * g(ii, jj - 1)) /
             (g(ii, jj) * (1.0 - feyp[jj - 1]) + g(ii, jj - 1) * feyp[jj - 1]);
    double gammas = gammai * gammad / (gammad * (1.0 - fexp[ii]) + gammai * fexp[ii]);
    gammai = g(ii, jj);
    gammad = g(ii + 1, jj);
    double di = deltaxp[ii], dd = deltaxp[ii + 1], ds = deltayv[jj - 1], dn = deltayv[jj];
    double deltax = deltaxu[ii], deltay = deltayu[jj];
    double temp_int = fexp[ii] * temp(ii + 1, jj) + (1.0 - fexp[ii]) * temp(ii, jj);
    AI(ii, jj) = -(gammai * deltay / di * plaw(ui * di / gammai) + dmax0(ui * deltay));
    AD(ii, jj) = -(gammad * deltay / dd * plaw(ud * dd / gammad) + dmax0(-ud * deltay));
    double BSo = -(gammas * deltax / ds * plaw(vs * ds / gammas) + dmax0(vs * deltax));
    double BNo = -(gamman * deltax / dn * plaw(vn * dn / gamman) + dmax0(-vn * deltax));
    AC(ii, jj) = (-AI(ii, jj) - AD(ii, jj) - BSo - BNo - deltax * deltay * flin_u(ii, jj) +
                  deltax * deltay / dt) / rel_vel;
    Rx(ii, jj) = -BSo * u(ii, jj - 1) - BNo * u(ii, jj + 1) -
                 deltax * deltay * Ri(ii, jj) * temp_int + deltax * deltay * fcon_u(ii, jj) +
                 deltax * deltay * u_ant(ii, jj) / dt + (pres(ii, jj) - pres(ii + 1, jj)) * deltay +
                 AC(ii, jj) * (1.0 - rel_vel) * u(ii, jj);
    au(ii, jj) = AC(ii, jj) * rel_vel;
  }

  // ensambla_velu_y, source/mod_ec_momento.f90:551-724, called at main.f90:427
  void velu_y(int jj, int ii) {
    A2& g = gamma_momen;
    double ud = fexu[ii] * u(ii + 1, jj) + (1.0 - fexu[ii]) * u(ii, jj);
    double ui = fexu[ii - 1] * u(ii, jj) + (1.0 - fexu[ii - 1]) * u(ii - 1, jj);
    double vn = fexp[ii] * v(ii + 1, jj) + (1.0 - fexp[ii]) * v(ii, jj);
    double vs = fexp[ii] * v(ii + 1, jj - 1) + (1.0 - fexp[ii]) * v(ii, jj - 1);
    double gammad = (g(ii + 1, jj + 1) * g(ii + 1, jj)) /
                    (g(ii + 1, jj + 1) * (1.0 - feyp[jj]) + g(ii + 1, jj) * feyp[jj]);
    double gammai = (g(ii, jj + 1) * g(ii, jj)) /
                    (g(ii, jj + 1) * (1.0 - feyp[jj]) + g(ii, jj) * feyp[jj]);
    double gamman = gammai * gammad / (gammad * (1.0 - fexp[ii]) + gammai * fexp[ii]);
    gammad = (g(ii + 1, jj) * g(ii + 1, jj - 1)) /
             (g(ii + 1, jj) * (1.0 - feyp[jj - 1]) + g(ii + 1, jj - 1) * feyp[jj - 1]);
    gammai = (g(ii, jj) * g(ii, jj - 1)) /
             (g(ii, jj) * (1.0 - feyp[jj - 1]) + g(ii, jj - 1) * feyp[jj - 1]);
    double gammas = gammai * gammad / (gammad * (1.0 - fexp[ii]) + gammai * fexp[ii]);
    gammai = g(ii, jj);
    gammad = g(ii + 1, jj);
    double di = deltaxp[ii], dd = deltaxp[ii + 1], ds = deltayv[jj - 1], dn = deltayv[jj];
    double deltax = deltaxu[ii], deltay = deltayu[jj];
    double temp_int = fexp[ii] * temp(ii + 1, jj) + (1.0 - fexp[ii]) * temp(ii, jj);
    double AIo = -(gammai * deltay / di * plaw(ui * di / gammai) + dmax0(ui * deltay));
    double ADo = -(gammad * deltay / dd * plaw(ud * dd / gammad) + dmax0(-ud * deltay));
    BS(jj, ii) = -(gammas * deltax / ds * plaw(vs * ds / gammas) + dmax0(vs * deltax));
    BN(jj, ii) = -(gamman * deltax / dn * plaw(vn * dn / gamman) + dmax0(-vn * deltax));
    BC(jj, ii) = (-AIo - ADo - BS(jj, ii) - BN(jj, ii) - deltax * deltay * flin_u(ii, jj) +
                  deltax * deltay / dt) / rel_vel;
    Ry(jj, ii) = -AIo * u(ii - 1, jj) - ADo * u(ii + 1, jj) -
                 deltax * deltay * Ri(ii, jj) * temp_int + deltax * deltay * fcon_u(ii, jj) +
                 deltax * deltay * u_ant(ii, jj) / dt + (pres(ii, jj) - pres(ii + 1, jj)) * deltay +
                 BC(jj, ii) * (1.0 - rel_vel) * u(ii, jj);
  }

  // v face velocities and diffusion coefficients shared by ensambla_velv_x
  // (source/mod_ec_momento.f90:818-874) and ensambla_velv_y (:1006-1062).
  struct VCoef { double AI, AD, BS, BN, temp_int; };
  VCoef velv_common(int ii, int jj) {
    A2& g = gamma_momen;
    double ud = feyp[jj] * u(ii, jj + 1) + (1.0 - feyp[jj]) * u(ii, jj);
    double ui = feyp[jj] * u(ii - 1, jj + 1) + (1.0 - feyp[jj]) * u(ii - 1, jj);
    double vn = feyv[jj] * v(ii, jj + 1) + (1.0 - feyv[jj]) * v(ii, jj);
    double vs = feyv[jj - 1] * v(ii, jj) + (1.0 - feyv[jj - 1]) * v(ii, jj - 1);
    double gammas = (g(ii + 1, jj) * g(ii, jj)) /
                    (g(ii + 1, jj) * (1.0 - fexp[ii]) + g(ii, jj) * fexp[ii]);
    double gamman = (g(ii + 1, jj + 1) * g(ii, jj + 1)) /
                    (g(ii + 1, jj + 1) * (1.0 - fexp[ii]) + g(ii, jj + 1) * fexp[ii]);
    double gammad = (gamman * gammas) / (gamman * (1.0 - feyp[jj]) + gammas * feyp[jj]);
    gammas = (g(ii, jj) * g(ii - 1, jj)) /
             (g(ii, jj) * (1.0 - fexp[ii - 1]) + g(ii - 1, jj) * fexp[ii - 1]);
    gamman = (g(ii, jj + 1) * g(ii - 1, jj + 1)) /
             (g(ii, jj + 1) * (1.0 - fexp[ii - 1]) + g(ii - 1, jj + 1) * fexp[ii - 1]);
    double gammai = (gammas * gamman) / (gamman * (1.0 - feyp[jj]) + gammas * feyp[jj]);
    gamman = g(ii, jj + 1);
    gammas = g(ii, jj);
    double di = deltaxu[ii - 1], dd = deltaxu[ii], ds = deltayp[jj], dn = deltayp[jj + 1];
    VCoef c;
    c.temp_int = feyp[jj] * temp(ii, jj + 1) + (1.0 - feyp[jj]) * temp(ii, jj);
    c.AI = -(gammai * deltayv[jj] / di * plaw(ui * di / gammai) + dmax0(ui * deltayv[jj]));
    c.AD = -(gammad * deltayv[jj] / dd * plaw(ud * dd / gammad) + dmax0(-ud * deltayv[jj]));
    c.BS = -(gammas * deltaxv[ii] / ds * plaw(vs * ds / gammas) + dmax0(vs * deltaxv[ii]));
    c.BN = -(gamman * deltaxv[ii] / dn * plaw(vn * dn / gamman) + dmax0(-vn * deltaxv[ii]));
    return c;
  }

  // ensambla_velv_x, source/mod_ec_momento.f90:736-913, called at main.f90:651
  void velv_x(int ii, int jj) {
    VCoef k = velv_common(ii, jj);
    double dxdy = deltaxv[ii] * deltayv[jj];
    AI(ii, jj) = k.AI;
    AD(ii, jj) = k.AD;
    AC(ii, jj) = (-AI(ii, jj) - AD(ii, jj) - k.BS - k.BN - dxdy * flin_v(ii, jj) + dxdy / dt) /
                 rel_vel;
    Rx(ii, jj) = -k.BS * v(ii, jj - 1) - k.BN * v(ii, jj + 1) - dxdy * Riy(ii, jj) * k.temp_int +
                 dxdy * fcon_v(ii, jj) + dxdy * v_ant(ii, jj) / dt +
                 (pres(ii, jj) - pres(ii, jj + 1)) * deltaxv[ii] +
                 AC(ii, jj) * (1.0 - rel_vel) * v(ii, jj);
    av(ii, jj) = AC(ii, jj) * rel_vel;
  }

  // ensambla_velv_y, source/mod_ec_momento.f90:925-1098, called at main.f90:574
  void velv_y(int jj, int ii) {
    VCoef k = velv_common(ii, jj);
    double dxdy = deltaxv[ii] * deltayv[jj];
    BS(jj, ii) = k.BS;
    BN(jj, ii) = k.BN;
    BC(jj, ii) = (-k.AI - k.AD - BS(jj, ii) - BN(jj, ii) - dxdy * flin_v(ii, jj) + dxdy / dt) /
                 rel_vel;
    Ry(jj, ii) = -k.AI * v(ii - 1, jj) - k.AD * v(ii + 1, jj) - dxdy * Riy(ii, jj) * k.temp_int +
                 dxdy * fcon_v(ii, jj) + dxdy * v_ant(ii, jj) / dt +
                 (pres(ii, jj) - pres(ii, jj + 1)) * deltaxv[ii] +
                 BC(jj, ii) * (1.0 - rel_vel) * v(ii, jj);
  }

  // Shared part of ensambla_energia_x/_y, source/mod_ec_energia.f90:213-259
  // and :380-426.  The dummies fexpo/feypo are bound to fexu/feyv by the calls.
  struct TCoef { double AI, AD, BS, BN; };
  TCoef energia_common(int ii, int jj) {
    A2& g = gamma_energ;
    const std::vector<double>& fx = fexu;  // dummy fexpo <- actual fexu (main.f90:990)
    const std::vector<double>& fy = feyv;  // dummy feypo <- actual feyv
    double ud = u(ii, jj), ui = u(ii - 1, jj), vn = v(ii, jj), vs = v(ii, jj - 1);
    double di = deltaxu[ii - 1], dd = deltaxu[ii], ds = deltayv[jj - 1], dn = deltayv[jj];
    double gammad = (g(ii + 1, jj) * g(ii, jj)) /
                    (g(ii + 1, jj) * (1.0 - fx[ii]) + g(ii, jj) * fx[ii]);
    double gammai = (g(ii, jj) * g(ii - 1, jj)) /
                    (g(ii, jj) * (1.0 - fx[ii - 1]) + g(ii - 1, jj) * fx[ii - 1]);
    double gamman = (g(ii, jj + 1) * g(ii, jj)) /
                    (g(ii, jj + 1) * (1.0 - fy[jj]) + g(ii, jj) * fy[jj]);
    double gammas = (g(ii, jj) * g(ii, jj - 1)) /
                    (g(ii, jj) * (1.0 - fy[jj - 1]) + g(ii, jj - 1) * fy[jj - 1]);
    TCoef c;
    c.AI = -(gammai * deltayp[jj] / di * plaw(ui * di / gammai) + dmax0(ui * deltayp[jj]));
    c.AD = -(gammad * deltayp[jj] / dd * plaw(ud * dd / gammad) + dmax0(-ud * deltayp[jj]));
    c.BS = -(gammas * deltaxp[ii] / ds * plaw(vs * ds / gammas) + dmax0(vs * deltaxp[ii]));
    c.BN = -(gamman * deltaxp[ii] / dn * plaw(vn * dn / gamman) + dmax0(-vn * deltaxp[ii]));
    return c;
  }

  // ensambla_energia_x, source/mod_ec_energia.f90:119-276, called at main.f90:1060
  void energia_x(int ii, int jj) {
    TCoef k = energia_common(ii, jj);
    double dxdy = deltaxp[ii] * deltayp[jj];
    AI(ii, jj) = k.AI;
    AD(ii, jj) = k.AD;
    AC(ii, jj) = (-AI(ii, jj) - AD(ii, jj) - k.BS - k.BN - dxdy * flin_t(ii, jj) + dxdy / dt) /
                 rel_ener;
    Rx(ii, jj) = -k.BS * temp(ii, jj - 1) - k.BN * temp(ii, jj + 1) + dxdy * fcon_t(ii, jj) +
                 dxdy * temp_ant(ii, jj) / dt + AC(ii, jj) * (1.0 - rel_ener) * temp(ii, jj);
  }

  // ensambla_energia_y, source/mod_ec_energia.f90:286-443, called at main.f90:989
  void energia_y(int jj, int ii) {
    TCoef k = energia_common(ii, jj);
    double dxdy = deltaxp[ii] * deltayp[jj];
    BS(jj, ii) = k.BS;
    BN(jj, ii) = k.BN;
    BC(jj, ii) = (-k.AI - k.AD - BS(jj, ii) - BN(jj, ii) - dxdy * flin_t(ii, jj) + dxdy / dt) /
                 rel_ener;
    Ry(jj, ii) = -k.AI * temp(ii - 1, jj) - k.AD * temp(ii + 1, jj) + dxdy * fcon_t(ii, jj) +
                 dxdy * temp_ant(ii, jj) / dt + BC(jj, ii) * (1.0 - rel_ener) * temp(ii, jj);
  }

  // ensambla_corr_pres_x, source/mod_ec_momento.f90:145-246, called at main.f90:836
  void corr_pres_x(int jj, int ii) {
    double ud = u(ii, jj), ui = u(ii - 1, jj), vn = v(ii, jj), vs = v(ii, jj - 1);
    double ai = au(ii - 1, jj), ad = au(ii, jj), as = av(ii, jj - 1), an = av(ii, jj);
    AI(ii, jj) = -deltayp[jj] * deltayp[jj] / ai;
    AD(ii, jj) = -deltayp[jj] * deltayp[jj] / ad;
    double BSo = -deltaxp[ii] * deltaxp[ii] / as;
    double BNo = -deltaxp[ii] * deltaxp[ii] / an;
    AC(ii, jj) = (-AI(ii, jj) - AD(ii, jj) - BSo - BNo) / rel_pres;
    b_o(ii, jj) = (ui - ud) * deltayp[jj] + (vs - vn) * deltaxp[ii];
    Rx(ii, jj) = -BSo * corr_pres(ii, jj - 1) - BNo * corr_pres(ii, jj + 1) + b_o(ii, jj) +
                 (1.0 - rel_pres) * AC(ii, jj) * corr_pres(ii, jj);
  }

  // ensambla_corr_pres_y, source/mod_ec_momento.f90:256-355, called at main.f90:777
  void corr_pres_y(int ii, int jj) {
    double ud = u(ii, jj), ui = u(ii - 1, jj), vn = v(ii, jj), vs = v(ii, jj - 1);
    double ai = au(ii - 1, jj), ad = au(ii, jj), as = av(ii, jj - 1), an = av(ii, jj);
    double AIo = -deltayp[jj] * deltayp[jj] / ai;
    double ADo = -deltayp[jj] * deltayp[jj] / ad;
    BS(jj, ii) = -deltaxp[ii] * deltaxp[ii] / as;
    BN(jj, ii) = -deltaxp[ii] * deltaxp[ii] / an;
    BC(jj, ii) = (-AIo - ADo - BS(jj, ii) - BN(jj, ii)) / rel_pres;
    double bo = (ui - ud) * deltayp[jj] + (vs - vn) * deltaxp[ii];
    Ry(jj, ii) = -AIo * corr_pres(ii - 1, jj) - ADo * corr_pres(ii + 1, jj) + bo +
                 (1.0 - rel_pres) * BC(jj, ii) * corr_pres(ii, jj);
  }

  // residuo_u, source/mod_ec_momento.f90:1107-1266, called at main.f90:1176.
  // Keeps the reference's numerator g(ii,jj+1)*g(ii,jj) in the south
  // auxiliary (:1208), which differs from ensambla_velu_x (:476).
  void residuo_u(int ii, int jj) {
    A2& g = gamma_momen;
    double ud = fexu[ii] * u(ii + 1, jj) + (1.0 - fexu[ii]) * u(ii, jj);
    double ui = fexu[ii - 1] * u(ii, jj) + (1.0 - fexu[ii - 1]) * u(ii - 1, jj);
    double vn = fexp[ii] * v(ii + 1, jj) + (1.0 - fexp[ii]) * v(ii, jj);
    double vs = fexp[ii] * v(ii + 1, jj - 1) + (1.0 - fexp[ii]) * v(ii, jj - 1);
    double gammad = (g(ii + 1, jj + 1) * g(ii + 1, jj)) /
                    (g(ii + 1, jj + 1) * (1.0 - feyp[jj]) + g(ii + 1, jj) * feyp[jj]);
    double gammai = (g(ii, jj + 1) * g(ii, jj)) /
                    (g(ii, jj + 1) * (1.0 - feyp[jj]) + g(ii, jj) * feyp[jj]);
    double gamman = gammai * gammad / (gammad * (1.0 - fexp[ii]) + gammai * fexp[ii]);
    gammad = (g(ii + 1, jj) * g(ii + 1, jj - 1)) /
             (g(ii + 1, jj) * (1.0 - feyp[jj - 1]) + g(ii + 1, jj - 1) * feyp[jj - 1]);
    gammai = (g(ii, jj + 1) * g(ii, jj)) /
             (g(ii, jj) * (1.0 - feyp[jj - 1]) + g(ii, jj - 1) * feyp[jj - 1]);
    double gammas = gammai * gammad / (gammad * (1.0 - fexp[ii]) + gammai * fexp[ii]);
    gammai = g(ii, jj);
    gammad = g(ii + 1, jj);
    double di = deltaxp[ii], dd = deltaxp[ii + 1], ds = deltayv[jj - 1], dn = deltayv[jj];
    double temp_int = fexp[ii] * temp(ii + 1, jj) + (1.0 - fexp[ii]) * temp(ii, jj);
    double AIo = (gammai * deltayu[jj] / di * plaw(ui * di / gammai) + dmax0(ui * deltayu[jj]));
    double ADo = (gammad * deltayu[jj] / dd * plaw(ud * dd / gammad) + dmax0(-ud * deltayu[jj]));
    double BSo = (gammas * deltaxu[ii] / ds * plaw(vs * ds / gammas) + dmax0(vs * deltaxu[ii]));
    double BNo = (gamman * deltaxu[ii] / dn * plaw(vn * dn / gamman) + dmax0(-vn * deltaxu[ii]));
    double dxdy = deltaxu[ii] * deltayu[jj];
    double ACo = AIo + ADo + BSo + BNo - deltaxu[ii] * deltayu[jj] * flin_u(ii, jj) + dxdy / dt;
    Resu(ii, jj) = AIo * u(ii - 1, jj) - ACo * u(ii, jj) + ADo * u(ii + 1, jj) +
                   BSo * u(ii, jj - 1) + BNo * u(ii, jj + 1) -
                   deltaxu[ii] * deltayu[jj] * Ri(ii, jj) * temp_int +
                   deltaxu[ii] * deltayu[jj] * fcon_u(ii, jj) +
                   deltaxu[ii] * deltayu[jj] * u_ant(ii, jj) / dt +
                   (pres(ii, jj) - pres(ii + 1, jj)) * deltayu[jj];
  }

  // impone_cond_frontera, source/mod_cond_frontera.f90:254-420.  Rows outside
  // the (mm,nn) / (kk,ll) shapes are skipped (the reference would write out of
  // bounds there).
  static void impone(const BCSide& cf, A2& AIo, A2& ACo, A2& ADo, A2& Rxo, int kk, int ll, A2* au_o) {
    int mm = AIo.n1, nn = AIo.n2;
    auto setrow = [&](int r, int jj, double a, double b, double c, double val) {
      if (r < 1 || r > mm || jj < 1 || jj > nn) return;
      AIo(r, jj) = a; ACo(r, jj) = b; ADo(r, jj) = c; Rxo(r, jj) = val;
    };
    auto setau = [&](int i, int j) {
      if (!au_o || i < 1 || i > au_o->n1 || j < 1 || j > au_o->n2) return;
      (*au_o)(i, j) = 1.e40;
    };
    for (int ldiv = 1; ldiv <= cf.ndivis; ++ldiv) {
      int t = cf.tipo[ldiv - 1];
      if (t != 1 && t != 2) continue;
      for (int jj = cf.indice[ldiv - 1]; jj <= cf.indice[ldiv]; ++jj) {
        const double val =
            (jj >= 1 && jj <= (int)cf.line_val.size()) ? cf.line_val[jj - 1] : cf.valor[ldiv - 1];
        switch (cf.lado) {
          case 'a':
            if (t == 1) setrow(1, jj, 0.0, 1.0, 0.0, val); else setrow(1, jj, 0.0, -1.0, 1.0, val);
            setau(1, jj);
            break;
          case 'b':
            if (t == 1) setrow(1, jj, 0.0, 1.0, 0.0, val); else setrow(1, jj, 0.0, -1.0, 1.0, val);
            setau(jj, 1);
            break;
          case 'c':
            if (t == 1) setrow(kk, jj, 0.0, 1.0, 0.0, val); else setrow(kk, jj, -1.0, 1.0, 0.0, val);
            setau(kk, jj);
            break;
          case 'd':
            if (t == 1) setrow(ll, jj, 0.0, 1.0, 0.0, val); else setrow(ll, jj, -1.0, 1.0, 0.0, val);
            setau(jj, ll);
            break;
          default: break;
        }
      }
    }
  }

  // ---------------------------------------------------------------------
  // Phases of ALGORITMO_SIMPLE (source/main.f90:395-1217)
  // ---------------------------------------------------------------------
  void phase_uy() {  // main.f90:420-484
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj)
      for (int ii = 2; ii <= mi - 1; ++ii) velu_y(jj, ii);
    impone(bcu[1], BS, BC, BN, Ry, mi, nj + 1, &au);
    impone(bcu[3], BS, BC, BN, Ry, mi, nj + 1, &au);
#pragma omp parallel for schedule(static)
    for (int ii = 2; ii <= mi - 1; ++ii) tridiagonal(BS.col(ii), BC.col(ii), BN.col(ii), Ry.col(ii), nj + 1);
#pragma omp parallel for schedule(static)
    for (int ii = 2; ii <= mi - 1; ++ii)
      for (int jj = 1; jj <= nj + 1; ++jj) u(ii, jj) = Ry(jj, ii);
  }
  void phase_ux() {  // main.f90:492-556
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj)
      for (int ii = 2; ii <= mi - 1; ++ii) velu_x(ii, jj);
    impone(bcu[0], AI, AC, AD, Rx, mi, nj + 1, &au);
    impone(bcu[2], AI, AC, AD, Rx, mi, nj + 1, &au);
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj) tridiagonal(AI.col(jj), AC.col(jj), AD.col(jj), Rx.col(jj), mi);
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj)
      for (int ii = 1; ii <= mi; ++ii) u(ii, jj) = Rx(ii, jj);
  }
  void phase_vy() {  // main.f90:570-640
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj - 1; ++jj)
      for (int ii = 2; ii <= mi; ++ii) velv_y(jj, ii);
    impone(bcv[1], BS, BC, BN, Ry, mi + 1, nj, &av);
    impone(bcv[3], BS, BC, BN, Ry, mi + 1, nj, &av);
#pragma omp parallel for schedule(static)
    for (int ii = 2; ii <= mi; ++ii) tridiagonal(BS.col(ii), BC.col(ii), BN.col(ii), Ry.col(ii), nj);
#pragma omp parallel for schedule(static)
    for (int ii = 2; ii <= mi; ++ii)
      for (int jj = 1; jj <= nj; ++jj) v(ii, jj) = Ry(jj, ii);
  }
  void phase_vx() {  // main.f90:647-711
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj - 1; ++jj)
      for (int ii = 2; ii <= mi; ++ii) velv_x(ii, jj);
    impone(bcv[0], AI, AC, AD, Rx, mi + 1, nj, &av);
    impone(bcv[2], AI, AC, AD, Rx, mi + 1, nj, &av);
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj - 1; ++jj) tridiagonal(AI.col(jj), AC.col(jj), AD.col(jj), Rx.col(jj), mi + 1);
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj - 1; ++jj)
      for (int ii = 1; ii <= mi + 1; ++ii) v(ii, jj) = Rx(ii, jj);
  }
  void phase_py() {  // main.f90:773-825
#pragma omp parallel for schedule(static)
    for (int ii = 2; ii <= mi; ++ii)
      for (int jj = 2; jj <= nj; ++jj) corr_pres_y(ii, jj);
    for (int ii = 2; ii <= mi; ++ii) {
      BC(1, ii) = 1.0; BN(1, ii) = 0.0; Ry(1, ii) = 0.0;
      BC(nj + 1, ii) = 1.0; BS(nj + 1, ii) = 0.0; Ry(nj + 1, ii) = 0.0;
    }
#pragma omp parallel for schedule(static)
    for (int ii = 2; ii <= mi; ++ii) tridiagonal(BS.col(ii), BC.col(ii), BN.col(ii), Ry.col(ii), nj + 1);
#pragma omp parallel for schedule(static)
    for (int ii = 2; ii <= mi; ++ii)
      for (int jj = 1; jj <= nj + 1; ++jj) corr_pres(ii, jj) = Ry(jj, ii);
  }
  void phase_px() {  // main.f90:832-879
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj)
      for (int ii = 2; ii <= mi; ++ii) corr_pres_x(jj, ii);
    for (int jj = 2; jj <= nj; ++jj) {
      AC(1, jj) = 1.0; AD(1, jj) = 0.0; Rx(1, jj) = 0.0;
      AI(mi + 1, jj) = 0.0; AC(mi + 1, jj) = 1.0; Rx(mi + 1, jj) = 0.0;
    }
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj) tridiagonal(AI.col(jj), AC.col(jj), AD.col(jj), Rx.col(jj), mi + 1);
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj)
      for (int ii = 1; ii <= mi + 1; ++ii) corr_pres(ii, jj) = Rx(ii, jj);
  }
  void phase_ty() {  // main.f90:985-1049
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj)
      for (int ii = 2; ii <= mi; ++ii) energia_y(jj, ii);
    impone(bct[1], BS, BC, BN, Ry, mi + 1, nj + 1, nullptr);
    impone(bct[3], BS, BC, BN, Ry, mi + 1, nj + 1, nullptr);
#pragma omp parallel for schedule(static)
    for (int ii = 2; ii <= mi; ++ii) tridiagonal(BS.col(ii), BC.col(ii), BN.col(ii), Ry.col(ii), nj + 1);
#pragma omp parallel for schedule(static)
    for (int ii = 2; ii <= mi; ++ii)
      for (int jj = 1; jj <= nj + 1; ++jj) temp(ii, jj) = Ry(jj, ii);
  }
  void phase_tx() {  // main.f90:1056-1121
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj)
      for (int ii = 2; ii <= mi; ++ii) energia_x(ii, jj);
    impone(bct[0], AI, AC, AD, Rx, mi + 1, nj + 1, nullptr);
    impone(bct[2], AI, AC, AD, Rx, mi + 1, nj + 1, nullptr);
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj) tridiagonal(AI.col(jj), AC.col(jj), AD.col(jj), Rx.col(jj), mi + 1);
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj)
      for (int ii = 1; ii <= mi + 1; ++ii) temp(ii, jj) = Rx(ii, jj);
  }
  void phase_correct() {  // main.f90:931-962
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj)
      for (int ii = 2; ii <= mi; ++ii) pres(ii, jj) = pres(ii, jj) + p_update * corr_pres(ii, jj);
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj - 1; ++jj)
      for (int ii = 2; ii <= mi - 1; ++ii) {
        u(ii, jj) = u(ii, jj) + deltayu[jj] * (corr_pres(ii, jj) - corr_pres(ii + 1, jj)) / au(ii, jj);
        v(ii, jj) = v(ii, jj) + deltaxv[ii] * (corr_pres(ii, jj) - corr_pres(ii, jj + 1)) / av(ii, jj);
      }
    for (int ii = 2; ii <= mi - 1; ++ii)
      u(ii, nj) = u(ii, nj) + deltayu[nj] * (corr_pres(ii, nj) - corr_pres(ii + 1, nj)) / au(ii, nj);
    for (int jj = 2; jj <= nj - 1; ++jj)
      v(mi, jj) = v(mi, jj) + deltaxv[mi] * (corr_pres(mi, jj) - corr_pres(mi, jj + 1)) / av(mi, jj);
  }
  void phase_residual() {  // main.f90:1169-1185
#pragma omp parallel for schedule(static)
    for (int jj = 2; jj <= nj; ++jj)
      for (int ii = 2; ii <= mi - 1; ++ii) residuo_u(ii, jj);
  }

  // Sum of squares over ii in [i0,i1], jj in [j0,j1]: per-jj partial sums in
  // parallel, then added in jj order (deterministic for any thread count).
  template <class F>
  double sumsq(int i0, int i1, int j0, int j1, F f) {
    if (j1 < j0) return 0.0;
    std::vector<double> part(j1 - j0 + 1, 0.0);
#pragma omp parallel for schedule(static)
    for (int jj = j0; jj <= j1; ++jj) {
      double s = 0.0;
      for (int ii = i0; ii <= i1; ++ii) { double d = f(ii, jj); s = s + d * d; }
      part[jj - j0] = s;
    }
    double s = 0.0;
    for (double p : part) s = s + p;
    return s;
  }

  // tridiagonal, source/mod_solucionador.f90:25-47 (in place: b clobbered, x in r)
  static void tridiagonal(double* a, double* b, double* c, double* r, int n) {
    for (int ii = 1; ii < n; ++ii) {
      r[ii] = r[ii] - (a[ii] / b[ii - 1]) * r[ii - 1];
      b[ii] = b[ii] - (a[ii] / b[ii - 1]) * c[ii - 1];
    }
    r[n - 1] = r[n - 1] / b[n - 1];
    for (int ii = n - 2; ii >= 0; --ii) r[ii] = (r[ii] - c[ii] * r[ii + 1]) / b[ii];
  }

  // One pass of the ALGORITMO_SIMPLE body (main.f90:404-1215).
  // Returns 0 = continue, 1 = converged exit, 2 = iteration-limit exit.
  int simple_body(bool outer_test) {
    // ecuacion_momento, main.f90:404-742
    for (;;) {
      fu.d = u.d;  // main.f90:406-411
      phase_uy();
      phase_ux();
      fv.d = v.d;  // main.f90:559-564
      phase_vy();
      phase_vx();
      double error = std::sqrt(sumsq(2, mi, 2, nj - 1, [&](int i, int j) { return v(i, j) - fv(i, j); }));
      err_u = error;
      ++n_momen;
      if (error < conv_u) { iter_ecuaci = 0; break; }
      else if (iter_ecuaci > iter_ecuaci_max) { iter_ecuaci = 0; break; }
      else iter_ecuaci = iter_ecuaci + 1;
    }
    // correccion_presion, main.f90:752-925
    corr_pres.fill(0.0);
    fcorr_pres.fill(0.0);
    for (;;) {
      for (int jj = 2; jj <= nj; ++jj)
        for (int ii = 2; ii <= mi; ++ii) fcorr_pres(ii, jj) = corr_pres(ii, jj);
      phase_py();
      phase_px();
      double error = std::sqrt(sumsq(2, mi, 2, nj, [&](int i, int j) { return corr_pres(i, j) - fcorr_pres(i, j); }));
      maxbo = std::sqrt(sumsq(2, mi, 2, nj, [&](int i, int j) { return b_o(i, j); }));
      err_p = error;
      ++n_pres;
      if (error < conv_p) { iter_ecuaci = 0; break; }
      else if (iter_ecuaci > iter_ecuaci_max) { iter_ecuaci = 0; break; }
      else iter_ecuaci = iter_ecuaci + 1;
    }
    phase_correct();
    // solucion_energia, main.f90:972-1158
    for (;;) {
      for (int jj = 2; jj <= nj; ++jj)
        for (int ii = 2; ii <= mi; ++ii) ftemp(ii, jj) = temp(ii, jj);
      phase_ty();
      phase_tx();
      double error = std::sqrt(sumsq(2, mi, 2, nj, [&](int i, int j) { return temp(i, j) - ftemp(i, j); }));
      err_t = error;
      ++n_ener;
      if (error < conv_t) { iter_ecuaci = 0; break; }
      else if (iter_ecuaci > iter_ecuaci_max) { iter_ecuaci = 0; break; }
      else iter_ecuaci = iter_ecuaci + 1;
    }
    // residuo, main.f90:1169-1199
    phase_residual();
    residuo = std::sqrt(sumsq(2, mi - 1, 2, nj, [&](int i, int j) { return Resu(i, j); }));
    ++n_simple;
    if (!outer_test) return 0;
    // main.f90:1202-1215
    if (maxbo < conv_paso && residuo < conv_resi) { iter_simple = 0; return 1; }
    else if (iter_simple > iter_simple_max) { iter_simple = 0; return 2; }
    else { iter_simple = iter_simple + 1; return 0; }
  }

  // time-step roll, main.f90:1251-1270
  void roll() {
    temp_ant.d = temp.d;
    u_ant.d = u.d;
    v_ant.d = v.d;
  }
};

// nusselt_promedio_y, source/mod_postproceso.f90:100-215.  Generalised to a
// wall in either direction: `along` are the coordinates along the wall
// (xp for the horizontal walls), `across` those normal to it (yp), and
// f(k, l) is T at along-index k, across-index l.  quirk = true keeps the
// reference rule that derivada is only evaluated on k0..k1 and is 0 beyond
// (read by the last panel); quirk = false (vertical-wall extension)
// evaluates it on every node the panels touch.
template <class F>
static int nusselt_wall(const std::vector<double>& along, int n_along, const std::vector<double>& across,
                        int n_across, int k0, int k1, F f, double* nu0, double* nu1, bool quirk) {
  if (k0 < 1 || k1 < k0) return 1;
  for (int k = k0; k <= k1; k += 2)
    if (k + 2 > n_along) return 1;
  std::vector<double> der(n_along + 1, 0.0);
  auto integrate = [&]() {
    double nu = 0.0;
    for (int ii = k0; ii <= k1; ii += 2) {
      double x_o = along[ii], x_1 = along[ii + 1], x_2 = along[ii + 2];
      double y_o = der[ii], y_1 = der[ii + 1], y_2 = der[ii + 2];
      double alpha = ((y_2 - y_1) / (x_2 - x_1) - (y_1 - y_o) / (x_1 - x_o)) / (x_2 - x_o);
      double beta = (y_2 - y_1) / (x_2 - x_1) - alpha * (x_1 + x_2);
      double gamma = y_o - alpha * x_o * x_o - beta * x_o;
      nu = nu + alpha / 3.0 * (x_2 * x_2 * x_2 - x_o * x_o * x_o) + beta / 2.0 * (x_2 * x_2 - x_o * x_o) +
           gamma * (x_2 - x_o);
    }
    return -nu;
  };
  const std::vector<double>& y = across;
  int kd = k1;
  if (!quirk) kd = std::min(k1 + 2, n_along);
  int jj = 1;
  for (int ii = k0; ii <= kd; ++ii) {
    double dy1 = f(ii, jj + 1) - f(ii, jj), dy2 = f(ii, jj + 2) - f(ii, jj + 1);
    double dx1 = y[jj + 1] - y[jj], dx2 = y[jj + 2] - y[jj + 1];
    double a = (dy2 / dx2 - dy1 / dx1) / (dx1 + dx2);
    double b = dy2 / dx2 - a * (y[jj + 1] + y[jj + 2]);
    der[ii] = 2.0 * a * y[jj] + b;
  }
  *nu0 = integrate();
  std::fill(der.begin(), der.end(), 0.0);
  jj = n_across - 2;
  for (int ii = k0; ii <= kd; ++ii) {
    double dy1 = f(ii, jj + 1) - f(ii, jj), dy2 = f(ii, jj + 2) - f(ii, jj + 1);
    double dx1 = y[jj + 1] - y[jj], dx2 = y[jj + 2] - y[jj + 1];
    double a = (dy2 / dx2 - dy1 / dx1) / (dx1 + dx2);
    double b = dy2 / dx2 - a * (y[jj + 1] + y[jj + 2]);
    der[ii] = 2.0 * a * y[jj + 2] + b;
  }
  *nu1 = integrate();
  return 0;
}

}  // namespace

// ------------------------------------------------------------------------
// C interface (ctypes).  All 2-D arrays are Fortran column-major with the
// reference shapes: u (mi,nj+1), v (mi+1,nj), p/T/p' (mi+1,nj+1).
// ------------------------------------------------------------------------
extern "C" {

struct ixo_case;

ixo_case* ixo_new(int mi, int nj) {
  if (mi < 4 || nj < 4) return nullptr;
  Case* c = new Case();
  c->alloc(mi, nj);
  return reinterpret_cast<ixo_case*>(c);
}
void ixo_free(ixo_case* h) { delete reinterpret_cast<Case*>(h); }

void ixo_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
int ixo_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int ixo_set_mesh(ixo_case* h, const double* xu, const double* yv, const double* xp, const double* yp) {
  Case& c = *reinterpret_cast<Case*>(h);
  for (int i = 1; i <= c.mi; ++i) c.xu[i] = xu[i - 1];
  for (int j = 1; j <= c.nj; ++j) c.yv[j] = yv[j - 1];
  for (int i = 1; i <= c.mi + 1; ++i) c.xp[i] = xp[i - 1];
  for (int j = 1; j <= c.nj + 1; ++j) c.yp[j] = yp[j - 1];
  c.metrics();
  return 0;
}

// d[]: gamma_momen, gamma_energ, Ri, Riy, dt, rel_vel, rel_pres, rel_ener,
//      conv_u, conv_p, conv_t, conv_resi, conv_paso, p_update
// n[]: iter_ecuaci_max, iter_simple_max
int ixo_set_params(ixo_case* h, const double* d, const int* n) {
  Case& c = *reinterpret_cast<Case*>(h);
  c.gamma_momen.fill(d[0]);
  c.gamma_energ.fill(d[1]);
  c.Ri.fill(d[2]);
  c.Riy.fill(d[3]);
  c.dt = d[4]; c.rel_vel = d[5]; c.rel_pres = d[6]; c.rel_ener = d[7];
  c.conv_u = d[8]; c.conv_p = d[9]; c.conv_t = d[10]; c.conv_resi = d[11]; c.conv_paso = d[12];
  c.p_update = d[13];
  c.iter_ecuaci_max = n[0];
  c.iter_simple_max = n[1];
  return 0;
}

// var 0=u 1=v 2=T; side 0..3 = a..d; tipo: 1 diri, 2 neum, 0 other;
// indice: ndivis+1 entries (1-based grid indices).
int ixo_set_bc(ixo_case* h, int var, int side, int ndivis, const int* tipo, const double* valor,
               const int* indice) {
  Case& c = *reinterpret_cast<Case*>(h);
  if (var < 0 || var > 2 || side < 0 || side > 3 || ndivis < 0 || ndivis > 15) return 1;
  BCSide* s = var == 0 ? c.bcu : var == 1 ? c.bcv : c.bct;
  BCSide& b = s[side];
  b = BCSide();
  b.ndivis = ndivis;
  b.lado = ndivis > 0 ? (char)('a' + side) : 'z';
  for (int k = 0; k < ndivis; ++k) { b.tipo[k] = tipo[k]; b.valor[k] = valor[k]; }
  for (int k = 0; k <= ndivis; ++k) b.indice[k] = indice[k];
  return 0;
}

// Per-line boundary values of one side (the extension of BCSide above), for
// the lines of that side in the variable's shape: sides a and c have nj+1
// lines for u and T and nj for v; sides b and d have mi for u and mi+1 for v
// and T.  Call after ixo_set_bc for the same side.
int ixo_set_bc_values(ixo_case* h, int var, int side, const double* values) {
  Case& c = *reinterpret_cast<Case*>(h);
  if (var < 0 || var > 2 || side < 0 || side > 3 || !values) return 1;
  const int mi = c.mi, nj = c.nj;
  const int nl = (side == 0 || side == 2) ? (var == 1 ? nj : nj + 1) : (var == 0 ? mi : mi + 1);
  BCSide* s = var == 0 ? c.bcu : var == 1 ? c.bcv : c.bct;
  s[side].line_val.assign(values, values + nl);
  return 0;
}

int ixo_set_sources(ixo_case* h, int var, const double* fcon, const double* flin) {
  Case& c = *reinterpret_cast<Case*>(h);
  A2* con = var == 0 ? &c.fcon_u : var == 1 ? &c.fcon_v : &c.fcon_t;
  A2* lin = var == 0 ? &c.flin_u : var == 1 ? &c.flin_v : &c.flin_t;
  if (fcon) std::memcpy(con->d.data(), fcon, con->d.size() * sizeof(double)); else con->fill(0.0);
  if (flin) std::memcpy(lin->d.data(), flin, lin->d.size() * sizeof(double)); else lin->fill(0.0);
  return 0;
}

static void cp_in(A2& a, const double* p) { if (p) std::memcpy(a.d.data(), p, a.d.size() * sizeof(double)); }
static void cp_out(A2& a, double* p) { if (p) std::memcpy(p, a.d.data(), a.d.size() * sizeof(double)); }

int ixo_set_state(ixo_case* h, const double* u, const double* v, const double* p, const double* T,
                  const double* u_ant, const double* v_ant, const double* T_ant) {
  Case& c = *reinterpret_cast<Case*>(h);
  cp_in(c.u, u); cp_in(c.v, v); cp_in(c.pres, p); cp_in(c.temp, T);
  cp_in(c.u_ant, u_ant); cp_in(c.v_ant, v_ant); cp_in(c.temp_ant, T_ant);
  return 0;
}
int ixo_get_state(ixo_case* h, double* u, double* v, double* p, double* T, double* u_ant, double* v_ant,
                  double* T_ant) {
  Case& c = *reinterpret_cast<Case*>(h);
  cp_out(c.u, u); cp_out(c.v, v); cp_out(c.pres, p); cp_out(c.temp, T);
  cp_out(c.u_ant, u_ant); cp_out(c.v_ant, v_ant); cp_out(c.temp_ant, T_ant);
  return 0;
}
int ixo_get_aux(ixo_case* h, double* au, double* av, double* b_o, double* resu, double* corr_pres) {
  Case& c = *reinterpret_cast<Case*>(h);
  cp_out(c.au, au); cp_out(c.av, av); cp_out(c.b_o, b_o); cp_out(c.Resu, resu); cp_out(c.corr_pres, corr_pres);
  return 0;
}

// report[]: maxbo, residuo, err_u, err_p, err_t, n_simple, n_momen, n_pres, n_ener, exit_code
static void fill_report(Case& c, double* rep, int code) {
  if (!rep) return;
  rep[0] = c.maxbo; rep[1] = c.residuo; rep[2] = c.err_u; rep[3] = c.err_p; rep[4] = c.err_t;
  rep[5] = (double)c.n_simple; rep[6] = (double)c.n_momen; rep[7] = (double)c.n_pres;
  rep[8] = (double)c.n_ener; rep[9] = code;
}

// Exactly n passes of the SIMPLE body, without the outer convergence test.
int ixo_simple_iterations(ixo_case* h, int n, double* report) {
  Case& c = *reinterpret_cast<Case*>(h);
  for (int k = 0; k < n; ++k) c.simple_body(false);
  fill_report(c, report, 0);
  return 0;
}

// The ALGORITMO_SIMPLE loop with the reference's exit logic (main.f90:1202-1215).
int ixo_simple_loop(ixo_case* h, double* report) {
  Case& c = *reinterpret_cast<Case*>(h);
  int code;
  while ((code = c.simple_body(true)) == 0) {}
  fill_report(c, report, code);
  return 0;
}

int ixo_roll(ixo_case* h) { reinterpret_cast<Case*>(h)->roll(); return 0; }

// One phase, for per-kernel parity checks: 0 uy, 1 ux, 2 vy, 3 vx, 4 py
// (p' neighbours read from the current corr_pres), 5 px, 6 correct, 7 ty,
// 8 tx, 9 residual.
int ixo_phase(ixo_case* h, int which) {
  Case& c = *reinterpret_cast<Case*>(h);
  switch (which) {
    case 0: c.phase_uy(); break;
    case 1: c.phase_ux(); break;
    case 2: c.phase_vy(); break;
    case 3: c.phase_vx(); break;
    case 4: c.phase_py(); break;
    case 5: c.phase_px(); break;
    case 6: c.phase_correct(); break;
    case 7: c.phase_ty(); break;
    case 8: c.phase_tx(); break;
    case 9: c.phase_residual(); break;
    default: return 1;
  }
  return 0;
}
int ixo_set_corr_pres(ixo_case* h, const double* cp) { cp_in(reinterpret_cast<Case*>(h)->corr_pres, cp); return 0; }
int ixo_set_auav(ixo_case* h, const double* au, const double* av) {
  Case& c = *reinterpret_cast<Case*>(h);
  cp_in(c.au, au); cp_in(c.av, av);
  return 0;
}

// Metric arrays (1-based Fortran arrays copied out 0-based): which 0..13 =
// deltaxp deltayp deltaxu deltayu deltaxv deltayv fexp feyp fexu feyv xu yv xp yp
int ixo_get_metric(ixo_case* h, int which, double* out) {
  Case& c = *reinterpret_cast<Case*>(h);
  std::vector<double>* m[] = {&c.deltaxp, &c.deltayp, &c.deltaxu, &c.deltayu, &c.deltaxv, &c.deltayv, &c.fexp,
                              &c.feyp, &c.fexu, &c.feyv, &c.xu, &c.yv, &c.xp, &c.yp};
  if (which < 0 || which > 13) return 1;
  std::vector<double>& v = *m[which];
  for (size_t k = 1; k < v.size(); ++k) out[k - 1] = v[k];
  return 0;
}

void ixo_tridiagonal(double* a, double* b, double* c, double* r, int n) { Case::tridiagonal(a, b, c, r, n); }

// Batch of independent systems, each contiguous (stride n), parallel over systems.
void ixo_tridiagonal_batch(double* a, double* b, double* c, double* r, int n, int nsys) {
#pragma omp parallel for schedule(static)
  for (int s = 0; s < nsys; ++s) {
    size_t o = (size_t)s * n;
    Case::tridiagonal(a + o, b + o, c + o, r + o, n);
  }
}

// nusselt_promedio_y (horizontal walls jj=1 and jj=nj+1), integrated over
// ii = i0..i1 step 2 (source/mod_postproceso.f90:100-215).
int ixo_nusselt_y(ixo_case* h, const double* T, int i0, int i1, double* nu0, double* nu1) {
  Case& c = *reinterpret_cast<Case*>(h);
  int ni = c.mi + 1, nj1 = c.nj + 1;
  auto f = [&](int k, int l) { return T[(size_t)(l - 1) * ni + (k - 1)]; };
  return nusselt_wall(c.xp, ni, c.yp, nj1, i0, i1, f, nu0, nu1, true);
}

// Vertical-wall counterpart (ii=1 and ii=mi+1), integrated over jj = j0..j1
// step 2: the same 3-point derivative and piecewise-quadratic integration,
// with the roles of x and y exchanged.  No counterpart in the reference.
int ixo_nusselt_x(ixo_case* h, const double* T, int j0, int j1, double* nu0, double* nu1) {
  Case& c = *reinterpret_cast<Case*>(h);
  int ni = c.mi + 1, nj1 = c.nj + 1;
  auto f = [&](int k, int l) { return T[(size_t)(k - 1) * ni + (l - 1)]; };
  return nusselt_wall(c.yp, nj1, c.xp, ni, j0, j1, f, nu0, nu1, false);
}

}  // extern "C"
