// ixb_device.cuh -- device-side data structures, coefficient assembly and
// line solvers of the SIMPLE hot path.
//
// Layout in HBM: every 2-D field (u, v, p, T, p', the *_ant copies, au, av,
// b_o, Resu, sources) is one array of (nj+2) rows x LD doubles, LD = mi+1
// rounded up to 32 elements (256 B), with Fortran index (ii,jj) at
// (jj-1)*LD + (ii-1).  Adjacent ii are adjacent in memory, so x-lines are
// contiguous and the y-lines of a tile of adjacent ii are read as coalesced
// row segments.  1-D metrics are 1-based arrays (element 0 unused).
//
// Arithmetic of the assembly follows the reference statements operand by
// operand (the library is built with -fmad=false), so the coefficients are
// bit-identical to the reference's IEEE evaluation.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ixb {

// metric arrays inside one device buffer, each `mstride` long, 1-based
enum Metric { M_DXP = 0, M_DYP, M_DXU, M_DYU, M_DXV, M_DYV, M_FEXP, M_FEYP, M_FEXU, M_FEYV, M_COUNT };

// sweeps: the eight line-solve phases of main.f90
enum Eq { EQ_UY = 0, EQ_UX, EQ_VY, EQ_VX, EQ_PY, EQ_PX, EQ_TY, EQ_TX, EQ_COUNT };

struct BCEntry {  // effective boundary row of one line (last covering segment wins)
  double val;
  int type;       // 0 none, 1 diri, 2 neum
  int pad;
};

struct NormSlot {        // deterministic two-level sum of squares
  double* partials;      // one per CTA
  unsigned int* counter; // CTAs finished (reset by the last one)
  double* result;        // sqrt(sum) written by the last CTA
};

template <class R>
struct Geo {
  int mi, nj, LD, mstride;
  const R* m;  // M_COUNT arrays
  R gm, ge, Ri, Riy, dt, rel_vel, rel_pres, rel_ener, p_update;
  __device__ __forceinline__ R met(int which, int k) const { return m[which * mstride + k]; }
  __device__ __forceinline__ size_t at(int ii, int jj) const { return (size_t)(jj - 1) * LD + (ii - 1); }
};

template <class R>
struct SweepIO {
  const R *u, *v, *T, *p, *pc;        // current fields (pc may be null: p' = 0)
  const R *u_ant, *v_ant, *T_ant;
  const R *au, *av;
  const R *fcon, *flin;               // sources of this equation (null: zero)
  const R* in;                        // swept field, current values (null: zero)
  R* out;                             // swept field, new values
  const R* prev;                      // field at the start of the inner pass (null: zero)
  R* aux;                             // au (u-x), av (v-x), b_o (p'-x)
  const BCEntry* bc_first;            // indexed by line
  const BCEntry* bc_last;
  NormSlot nrm0;                      // ||out - prev|| over interior rows of solved lines
  NormSlot nrm1;                      // ||b_o|| (p'-x)
  int m, mp;                          // rows per lane chunk, padded chunk pitch
};

template <class R>
struct Row { R a, b, c, d; };

// DMAX1(0, (1 - 0.1|P|)**5): the integer power as binary powering x*((x*x)*(x*x))
template <class R>
__device__ __forceinline__ R plaw(R pe) {
  R t = R(1) - R(0.1) * fabs(pe);
  R t2 = t * t;
  R t5 = t * (t2 * t2);
  return fmax(R(0), t5);
}
template <class R>
__device__ __forceinline__ R dmax0(R x) { return fmax(R(0), x); }

// harmonic face interpolation g1*g2/(g1*(1-f)+g2*f) of the reference
// (e.g. source/mod_ec_momento.f90:462-465) with its operand order
template <class R>
__device__ __forceinline__ R hmean(R g1, R g2, R f) {
  return (g1 * g2) / (g1 * (R(1) - f) + g2 * f);
}

// ---------------------------------------------------------------------------
// u momentum (ensambla_velu_x/_y, source/mod_ec_momento.f90:365-724)
// ---------------------------------------------------------------------------
template <class R>
struct UParts { R AI, AD, BS, BN, dxdy, tail; };

// Everything of the u row except the in-line/cross-line arrangement.
// `tail` = - dxdy*Ri*T_int + dxdy*fcon + dxdy*u_ant/dt + (p_P - p_E)*dy
// is NOT formed here because the reference adds it after the cross terms;
// the caller adds the terms in the reference order.
template <class R>
__device__ __forceinline__ void u_parts(const Geo<R>& G, const SweepIO<R>& io, const R* u, int ii, int jj,
                                        R& AI, R& AD, R& BS, R& BN, R& deltax, R& deltay, R& temp_int) {
  const R* v = io.v;
  const R fexu_i = G.met(M_FEXU, ii), fexu_m = G.met(M_FEXU, ii - 1);
  const R fexp_i = G.met(M_FEXP, ii);
  const R feyp_j = G.met(M_FEYP, jj), feyp_m = G.met(M_FEYP, jj - 1);
  R ud = fexu_i * u[G.at(ii + 1, jj)] + (R(1) - fexu_i) * u[G.at(ii, jj)];
  R ui = fexu_m * u[G.at(ii, jj)] + (R(1) - fexu_m) * u[G.at(ii - 1, jj)];
  R vn = fexp_i * v[G.at(ii + 1, jj)] + (R(1) - fexp_i) * v[G.at(ii, jj)];
  R vs = fexp_i * v[G.at(ii + 1, jj - 1)] + (R(1) - fexp_i) * v[G.at(ii, jj - 1)];
  const R g = G.gm;  // gamma_momen is uniform (main.f90:226, :238)
  R gammad = hmean(g, g, feyp_j);
  R gammai = hmean(g, g, feyp_j);
  R gamman = gammai * gammad / (gammad * (R(1) - fexp_i) + gammai * fexp_i);
  gammad = hmean(g, g, feyp_m);
  gammai = hmean(g, g, feyp_m);
  R gammas = gammai * gammad / (gammad * (R(1) - fexp_i) + gammai * fexp_i);
  gammai = g;
  gammad = g;
  R di = G.met(M_DXP, ii), dd = G.met(M_DXP, ii + 1), ds = G.met(M_DYV, jj - 1), dn = G.met(M_DYV, jj);
  deltax = G.met(M_DXU, ii);
  deltay = G.met(M_DYU, jj);
  temp_int = fexp_i * io.T[G.at(ii + 1, jj)] + (R(1) - fexp_i) * io.T[G.at(ii, jj)];
  AI = -(gammai * deltay / di * plaw(ui * di / gammai) + dmax0(ui * deltay));
  AD = -(gammad * deltay / dd * plaw(ud * dd / gammad) + dmax0(-ud * deltay));
  BS = -(gammas * deltax / ds * plaw(vs * ds / gammas) + dmax0(vs * deltax));
  BN = -(gamman * deltax / dn * plaw(vn * dn / gamman) + dmax0(-vn * deltax));
}

// X form (ensambla_velu_x): a=AI c=AD b=AC d=Rx, aux = au = AC*rel
template <class R>
__device__ __forceinline__ Row<R> assemble_ux(const Geo<R>& G, const SweepIO<R>& io, int ii, int jj, R& au) {
  const R* u = io.in;
  R AI, AD, BS, BN, dx, dy, tint;
  u_parts(G, io, u, ii, jj, AI, AD, BS, BN, dx, dy, tint);
  const size_t c0 = G.at(ii, jj);
  const R flin = io.flin ? io.flin[c0] : R(0);
  const R fcon = io.fcon ? io.fcon[c0] : R(0);
  Row<R> r;
  r.a = AI;
  r.c = AD;
  r.b = (-AI - AD - BS - BN - dx * dy * flin + dx * dy / G.dt) / G.rel_vel;
  r.d = -BS * u[G.at(ii, jj - 1)] - BN * u[G.at(ii, jj + 1)] - dx * dy * G.Ri * tint + dx * dy * fcon +
        dx * dy * io.u_ant[c0] / G.dt + (io.p[c0] - io.p[G.at(ii + 1, jj)]) * dy +
        r.b * (R(1) - G.rel_vel) * u[c0];
  au = r.b * G.rel_vel;
  return r;
}

// Y form (ensambla_velu_y): a=BS c=BN b=BC d=Ry
template <class R>
__device__ __forceinline__ Row<R> assemble_uy(const Geo<R>& G, const SweepIO<R>& io, int ii, int jj) {
  const R* u = io.in;
  R AI, AD, BS, BN, dx, dy, tint;
  u_parts(G, io, u, ii, jj, AI, AD, BS, BN, dx, dy, tint);
  const size_t c0 = G.at(ii, jj);
  const R flin = io.flin ? io.flin[c0] : R(0);
  const R fcon = io.fcon ? io.fcon[c0] : R(0);
  Row<R> r;
  r.a = BS;
  r.c = BN;
  r.b = (-AI - AD - BS - BN - dx * dy * flin + dx * dy / G.dt) / G.rel_vel;
  r.d = -AI * u[G.at(ii - 1, jj)] - AD * u[G.at(ii + 1, jj)] - dx * dy * G.Ri * tint + dx * dy * fcon +
        dx * dy * io.u_ant[c0] / G.dt + (io.p[c0] - io.p[G.at(ii + 1, jj)]) * dy +
        r.b * (R(1) - G.rel_vel) * u[c0];
  return r;
}

// ---------------------------------------------------------------------------
// v momentum (ensambla_velv_x/_y, source/mod_ec_momento.f90:736-1098)
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ void v_parts(const Geo<R>& G, const SweepIO<R>& io, const R* v, int ii, int jj,
                                        R& AI, R& AD, R& BS, R& BN, R& temp_int) {
  const R* u = io.u;
  const R feyp_j = G.met(M_FEYP, jj);
  const R feyv_j = G.met(M_FEYV, jj), feyv_m = G.met(M_FEYV, jj - 1);
  const R fexp_i = G.met(M_FEXP, ii), fexp_m = G.met(M_FEXP, ii - 1);
  R ud = feyp_j * u[G.at(ii, jj + 1)] + (R(1) - feyp_j) * u[G.at(ii, jj)];
  R ui = feyp_j * u[G.at(ii - 1, jj + 1)] + (R(1) - feyp_j) * u[G.at(ii - 1, jj)];
  R vn = feyv_j * v[G.at(ii, jj + 1)] + (R(1) - feyv_j) * v[G.at(ii, jj)];
  R vs = feyv_m * v[G.at(ii, jj)] + (R(1) - feyv_m) * v[G.at(ii, jj - 1)];
  const R g = G.gm;
  R gammas = hmean(g, g, fexp_i);
  R gamman = hmean(g, g, fexp_i);
  R gammad = (gamman * gammas) / (gamman * (R(1) - feyp_j) + gammas * feyp_j);
  gammas = hmean(g, g, fexp_m);
  gamman = hmean(g, g, fexp_m);
  R gammai = (gammas * gamman) / (gamman * (R(1) - feyp_j) + gammas * feyp_j);
  gamman = g;
  gammas = g;
  R di = G.met(M_DXU, ii - 1), dd = G.met(M_DXU, ii), ds = G.met(M_DYP, jj), dn = G.met(M_DYP, jj + 1);
  const R dyv = G.met(M_DYV, jj), dxv = G.met(M_DXV, ii);
  temp_int = feyp_j * io.T[G.at(ii, jj + 1)] + (R(1) - feyp_j) * io.T[G.at(ii, jj)];
  AI = -(gammai * dyv / di * plaw(ui * di / gammai) + dmax0(ui * dyv));
  AD = -(gammad * dyv / dd * plaw(ud * dd / gammad) + dmax0(-ud * dyv));
  BS = -(gammas * dxv / ds * plaw(vs * ds / gammas) + dmax0(vs * dxv));
  BN = -(gamman * dxv / dn * plaw(vn * dn / gamman) + dmax0(-vn * dxv));
}

template <class R>
__device__ __forceinline__ Row<R> assemble_vx(const Geo<R>& G, const SweepIO<R>& io, int ii, int jj, R& av) {
  const R* v = io.in;
  R AI, AD, BS, BN, tint;
  v_parts(G, io, v, ii, jj, AI, AD, BS, BN, tint);
  const size_t c0 = G.at(ii, jj);
  const R dxv = G.met(M_DXV, ii), dyv = G.met(M_DYV, jj);
  const R dxdy = dxv * dyv;
  const R flin = io.flin ? io.flin[c0] : R(0);
  const R fcon = io.fcon ? io.fcon[c0] : R(0);
  Row<R> r;
  r.a = AI;
  r.c = AD;
  r.b = (-AI - AD - BS - BN - dxdy * flin + dxdy / G.dt) / G.rel_vel;
  r.d = -BS * v[G.at(ii, jj - 1)] - BN * v[G.at(ii, jj + 1)] - dxdy * G.Riy * tint + dxdy * fcon +
        dxdy * io.v_ant[c0] / G.dt + (io.p[c0] - io.p[G.at(ii, jj + 1)]) * dxv +
        r.b * (R(1) - G.rel_vel) * v[c0];
  av = r.b * G.rel_vel;
  return r;
}

template <class R>
__device__ __forceinline__ Row<R> assemble_vy(const Geo<R>& G, const SweepIO<R>& io, int ii, int jj) {
  const R* v = io.in;
  R AI, AD, BS, BN, tint;
  v_parts(G, io, v, ii, jj, AI, AD, BS, BN, tint);
  const size_t c0 = G.at(ii, jj);
  const R dxv = G.met(M_DXV, ii), dyv = G.met(M_DYV, jj);
  const R dxdy = dxv * dyv;
  const R flin = io.flin ? io.flin[c0] : R(0);
  const R fcon = io.fcon ? io.fcon[c0] : R(0);
  Row<R> r;
  r.a = BS;
  r.c = BN;
  r.b = (-AI - AD - BS - BN - dxdy * flin + dxdy / G.dt) / G.rel_vel;
  r.d = -AI * v[G.at(ii - 1, jj)] - AD * v[G.at(ii + 1, jj)] - dxdy * G.Riy * tint + dxdy * fcon +
        dxdy * io.v_ant[c0] / G.dt + (io.p[c0] - io.p[G.at(ii, jj + 1)]) * dxv +
        r.b * (R(1) - G.rel_vel) * v[c0];
  return r;
}

// ---------------------------------------------------------------------------
// energy (ensambla_energia_x/_y, source/mod_ec_energia.f90:119-443).  The
// calls in main.f90:989 and :1060 bind fexu/feyv to the dummies fexpo/feypo.
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ void t_parts(const Geo<R>& G, const SweepIO<R>& io, int ii, int jj, R& AI, R& AD,
                                        R& BS, R& BN) {
  const R ud = io.u[G.at(ii, jj)], ui = io.u[G.at(ii - 1, jj)];
  const R vn = io.v[G.at(ii, jj)], vs = io.v[G.at(ii, jj - 1)];
  const R di = G.met(M_DXU, ii - 1), dd = G.met(M_DXU, ii), ds = G.met(M_DYV, jj - 1), dn = G.met(M_DYV, jj);
  const R g = G.ge;
  const R gammad = hmean(g, g, G.met(M_FEXU, ii));
  const R gammai = hmean(g, g, G.met(M_FEXU, ii - 1));
  const R gamman = hmean(g, g, G.met(M_FEYV, jj));
  const R gammas = hmean(g, g, G.met(M_FEYV, jj - 1));
  const R dyp = G.met(M_DYP, jj), dxp = G.met(M_DXP, ii);
  AI = -(gammai * dyp / di * plaw(ui * di / gammai) + dmax0(ui * dyp));
  AD = -(gammad * dyp / dd * plaw(ud * dd / gammad) + dmax0(-ud * dyp));
  BS = -(gammas * dxp / ds * plaw(vs * ds / gammas) + dmax0(vs * dxp));
  BN = -(gamman * dxp / dn * plaw(vn * dn / gamman) + dmax0(-vn * dxp));
}

template <class R>
__device__ __forceinline__ Row<R> assemble_tx(const Geo<R>& G, const SweepIO<R>& io, int ii, int jj) {
  const R* T = io.in;
  R AI, AD, BS, BN;
  t_parts(G, io, ii, jj, AI, AD, BS, BN);
  const size_t c0 = G.at(ii, jj);
  const R dxdy = G.met(M_DXP, ii) * G.met(M_DYP, jj);
  const R flin = io.flin ? io.flin[c0] : R(0);
  const R fcon = io.fcon ? io.fcon[c0] : R(0);
  Row<R> r;
  r.a = AI;
  r.c = AD;
  r.b = (-AI - AD - BS - BN - dxdy * flin + dxdy / G.dt) / G.rel_ener;
  r.d = -BS * T[G.at(ii, jj - 1)] - BN * T[G.at(ii, jj + 1)] + dxdy * fcon + dxdy * io.T_ant[c0] / G.dt +
        r.b * (R(1) - G.rel_ener) * T[c0];
  return r;
}

template <class R>
__device__ __forceinline__ Row<R> assemble_ty(const Geo<R>& G, const SweepIO<R>& io, int ii, int jj) {
  const R* T = io.in;
  R AI, AD, BS, BN;
  t_parts(G, io, ii, jj, AI, AD, BS, BN);
  const size_t c0 = G.at(ii, jj);
  const R dxdy = G.met(M_DXP, ii) * G.met(M_DYP, jj);
  const R flin = io.flin ? io.flin[c0] : R(0);
  const R fcon = io.fcon ? io.fcon[c0] : R(0);
  Row<R> r;
  r.a = BS;
  r.c = BN;
  r.b = (-AI - AD - BS - BN - dxdy * flin + dxdy / G.dt) / G.rel_ener;
  r.d = -AI * T[G.at(ii - 1, jj)] - AD * T[G.at(ii + 1, jj)] + dxdy * fcon + dxdy * io.T_ant[c0] / G.dt +
        r.b * (R(1) - G.rel_ener) * T[c0];
  return r;
}

// ---------------------------------------------------------------------------
// pressure correction (ensambla_corr_pres_x/_y, source/mod_ec_momento.f90:145-355)
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ R pc_at(const SweepIO<R>& io, const Geo<R>& G, int ii, int jj) {
  return io.in ? io.in[G.at(ii, jj)] : R(0);
}

template <class R>
__device__ __forceinline__ Row<R> assemble_px(const Geo<R>& G, const SweepIO<R>& io, int ii, int jj, R& bo) {
  const size_t c0 = G.at(ii, jj);
  const R ud = io.u[c0], ui = io.u[G.at(ii - 1, jj)], vn = io.v[c0], vs = io.v[G.at(ii, jj - 1)];
  const R ai = io.au[G.at(ii - 1, jj)], ad = io.au[c0], as = io.av[G.at(ii, jj - 1)], an = io.av[c0];
  const R dyp = G.met(M_DYP, jj), dxp = G.met(M_DXP, ii);
  Row<R> r;
  r.a = -dyp * dyp / ai;
  r.c = -dyp * dyp / ad;
  const R BS = -dxp * dxp / as;
  const R BN = -dxp * dxp / an;
  r.b = (-r.a - r.c - BS - BN) / G.rel_pres;
  bo = (ui - ud) * dyp + (vs - vn) * dxp;
  r.d = -BS * pc_at(io, G, ii, jj - 1) - BN * pc_at(io, G, ii, jj + 1) + bo +
        (R(1) - G.rel_pres) * r.b * pc_at(io, G, ii, jj);
  return r;
}

template <class R>
__device__ __forceinline__ Row<R> assemble_py(const Geo<R>& G, const SweepIO<R>& io, int ii, int jj) {
  const size_t c0 = G.at(ii, jj);
  const R ud = io.u[c0], ui = io.u[G.at(ii - 1, jj)], vn = io.v[c0], vs = io.v[G.at(ii, jj - 1)];
  const R ai = io.au[G.at(ii - 1, jj)], ad = io.au[c0], as = io.av[G.at(ii, jj - 1)], an = io.av[c0];
  const R dyp = G.met(M_DYP, jj), dxp = G.met(M_DXP, ii);
  const R AI = -dyp * dyp / ai;
  const R AD = -dyp * dyp / ad;
  Row<R> r;
  r.a = -dxp * dxp / as;
  r.c = -dxp * dxp / an;
  r.b = (-AI - AD - r.a - r.c) / G.rel_pres;
  const R bo = (ui - ud) * dyp + (vs - vn) * dxp;
  r.d = -AI * pc_at(io, G, ii - 1, jj) - AD * pc_at(io, G, ii + 1, jj) + bo +
        (R(1) - G.rel_pres) * r.b * pc_at(io, G, ii, jj);
  return r;
}

// ---------------------------------------------------------------------------
// u residual (residuo_u, source/mod_ec_momento.f90:1107-1266).  With a
// uniform gamma the reference's different south numerator (:1208) has the
// same value as in ensambla_velu_x.
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ R residual_u(const Geo<R>& G, const R* u, const R* v, const R* T, const R* p,
                                        const R* u_ant, const R* fcon, const R* flin, int ii, int jj) {
  const R fexu_i = G.met(M_FEXU, ii), fexu_m = G.met(M_FEXU, ii - 1);
  const R fexp_i = G.met(M_FEXP, ii);
  const R feyp_j = G.met(M_FEYP, jj), feyp_m = G.met(M_FEYP, jj - 1);
  R ud = fexu_i * u[G.at(ii + 1, jj)] + (R(1) - fexu_i) * u[G.at(ii, jj)];
  R ui = fexu_m * u[G.at(ii, jj)] + (R(1) - fexu_m) * u[G.at(ii - 1, jj)];
  R vn = fexp_i * v[G.at(ii + 1, jj)] + (R(1) - fexp_i) * v[G.at(ii, jj)];
  R vs = fexp_i * v[G.at(ii + 1, jj - 1)] + (R(1) - fexp_i) * v[G.at(ii, jj - 1)];
  const R g = G.gm;
  R gammad = hmean(g, g, feyp_j);
  R gammai = hmean(g, g, feyp_j);
  R gamman = gammai * gammad / (gammad * (R(1) - fexp_i) + gammai * fexp_i);
  gammad = hmean(g, g, feyp_m);
  gammai = hmean(g, g, feyp_m);
  R gammas = gammai * gammad / (gammad * (R(1) - fexp_i) + gammai * fexp_i);
  gammai = g;
  gammad = g;
  R di = G.met(M_DXP, ii), dd = G.met(M_DXP, ii + 1), ds = G.met(M_DYV, jj - 1), dn = G.met(M_DYV, jj);
  const R dxu = G.met(M_DXU, ii), dyu = G.met(M_DYU, jj);
  const size_t c0 = G.at(ii, jj);
  R temp_int = fexp_i * T[G.at(ii + 1, jj)] + (R(1) - fexp_i) * T[c0];
  R AI = (gammai * dyu / di * plaw(ui * di / gammai) + dmax0(ui * dyu));
  R AD = (gammad * dyu / dd * plaw(ud * dd / gammad) + dmax0(-ud * dyu));
  R BS = (gammas * dxu / ds * plaw(vs * ds / gammas) + dmax0(vs * dxu));
  R BN = (gamman * dxu / dn * plaw(vn * dn / gamman) + dmax0(-vn * dxu));
  const R fl = flin ? flin[c0] : R(0);
  const R fc = fcon ? fcon[c0] : R(0);
  R AC = AI + AD + BS + BN - dxu * dyu * fl + dxu * dyu / G.dt;
  return AI * u[G.at(ii - 1, jj)] - AC * u[c0] + AD * u[G.at(ii + 1, jj)] + BS * u[G.at(ii, jj - 1)] +
         BN * u[G.at(ii, jj + 1)] - dxu * dyu * G.Ri * temp_int + dxu * dyu * fc + dxu * dyu * u_ant[c0] / G.dt +
         (p[c0] - p[G.at(ii + 1, jj)]) * dyu;
}

// ---------------------------------------------------------------------------
// Line solvers on a line staged in shared memory.
// Row r of the (padded) line lives in chunk lane = r / m at slot r % m;
// arrays are [32][mp] with mp odd, so the 32 lanes walking their chunks
// hit distinct banks.
// ---------------------------------------------------------------------------

// Sequential Thomas, one thread, the exact operation order of
// tridiagonal (source/mod_solucionador.f90:25-47).  Solution left in sd.
template <class R>
__device__ void thomas_exact(R* sa, R* sb, R* sc, R* sd, int n, int m, int mp) {
  int lane = 0, k = 0;
  int prev = 0;  // offset of row i-1
  for (int i = 1; i < n; ++i) {
    if (++k == m) { k = 0; ++lane; }
    const int o = lane * mp + k;
    const R q = sa[o] / sb[prev];
    sd[o] = sd[o] - q * sd[prev];
    sb[o] = sb[o] - q * sc[prev];
    prev = o;
  }
  sd[prev] = sd[prev] / sb[prev];
  int nxt = prev;
  for (int i = n - 2; i >= 0; --i) {
    if (--k < 0) { k = m - 1; --lane; }
    const int o = lane * mp + k;
    sd[o] = (sd[o] - sc[o] * sd[nxt]) / sb[o];
    nxt = o;
  }
}

template <class R>
__device__ __forceinline__ R shfl_up_r(R x, int d) { return __shfl_up_sync(0xffffffffu, x, d); }
template <class R>
__device__ __forceinline__ R shfl_dn_r(R x, int d) { return __shfl_down_sync(0xffffffffu, x, d); }

// One warp per line: every lane eliminates its chunk of m >= 3 rows down to
// two rows coupled to the neighbouring chunks (forward and backward
// "modified Thomas" sweeps), the warp solves the 64-row reduced system by
// parallel cyclic reduction with register shuffles, and every lane
// back-substitutes its chunk.  (Thomas-PCR hybrid of Laszlo, Giles and
// Appleyard, ACM TOMS 42(4) 2016.)  Must be called by all 32 lanes.
template <class R>
__device__ void thomas_pcr_warp(R* sa, R* sb, R* sc, R* sd, int m, int mp) {
  const int lane = threadIdx.x & 31;
  R* a = sa + lane * mp;
  R* b = sb + lane * mp;
  R* c = sc + lane * mp;
  R* d = sd + lane * mp;
  // forward: rows 1..m-1 -> x_k + a'_k x_0 + c'_k x_{k+1} = d'_k
  const R a0 = a[0], b0 = b[0], c0 = c[0], d0 = d[0];
  R inv = R(1) / b[1];
  R ap = a[1] * inv, cp = c[1] * inv, dp = d[1] * inv;
  a[1] = ap; c[1] = cp; d[1] = dp;
  for (int k = 2; k < m; ++k) {
    const R ak = a[k];
    const R r = R(1) / (b[k] - ak * cp);
    ap = -ak * ap * r;
    dp = (d[k] - ak * dp) * r;
    cp = c[k] * r;
    a[k] = ap; c[k] = cp; d[k] = dp;
  }
  // reduced row 2*lane+1 (chunk's last row): x_{m-1} + ap x_0 + cp x_m = dp
  R oA = ap, oB = R(1), oC = cp, oD = dp;
  // backward: rows m-3..1 -> x_k + a''_k x_0 + c''_k x_{m-1} = d''_k
  R an = a[m - 2], cn = c[m - 2], dn = d[m - 2];
  for (int k = m - 3; k >= 1; --k) {
    const R ck = c[k];
    dn = d[k] - ck * dn;
    an = a[k] - ck * an;
    cn = -ck * cn;
    a[k] = an; c[k] = cn; d[k] = dn;
  }
  // reduced row 2*lane (chunk's first row): x_0 + A x_{-1} + C x_{m-1} = D
  const R r0 = R(1) / (b0 - c0 * an);
  R eA = a0 * r0, eB = R(1), eC = -c0 * cn * r0, eD = (d0 - c0 * dn) * r0;

  // PCR on the 64 interleaved rows (even = first rows, odd = last rows)
  {  // stride 1: even row needs odd of lane-1 and own odd; odd needs own even and even of lane+1
    R lA = shfl_up_r(oA, 1), lB = shfl_up_r(oB, 1), lC = shfl_up_r(oC, 1), lD = shfl_up_r(oD, 1);
    R hA = shfl_dn_r(eA, 1), hB = shfl_dn_r(eB, 1), hC = shfl_dn_r(eC, 1), hD = shfl_dn_r(eD, 1);
    if (lane == 0) { lA = R(0); lB = R(1); lC = R(0); lD = R(0); }
    if (lane == 31) { hA = R(0); hB = R(1); hC = R(0); hD = R(0); }
    const R k1e = eA / lB, k2e = eC / oB;
    const R k1o = oA / eB, k2o = oC / hB;
    const R nEA = -lA * k1e, nEB = eB - lC * k1e - oA * k2e, nEC = -oC * k2e, nED = eD - lD * k1e - oD * k2e;
    const R nOA = -eA * k1o, nOB = oB - eC * k1o - hA * k2o, nOC = -hC * k2o, nOD = oD - eD * k1o - hD * k2o;
    eA = nEA; eB = nEB; eC = nEC; eD = nED;
    oA = nOA; oB = nOB; oC = nOC; oD = nOD;
  }
#pragma unroll
  for (int dl = 1; dl < 32; dl <<= 1) {  // row stride 2*dl: same-parity rows of lanes +-dl
    R lEA = shfl_up_r(eA, dl), lEB = shfl_up_r(eB, dl), lEC = shfl_up_r(eC, dl), lED = shfl_up_r(eD, dl);
    R hEA = shfl_dn_r(eA, dl), hEB = shfl_dn_r(eB, dl), hEC = shfl_dn_r(eC, dl), hED = shfl_dn_r(eD, dl);
    R lOA = shfl_up_r(oA, dl), lOB = shfl_up_r(oB, dl), lOC = shfl_up_r(oC, dl), lOD = shfl_up_r(oD, dl);
    R hOA = shfl_dn_r(oA, dl), hOB = shfl_dn_r(oB, dl), hOC = shfl_dn_r(oC, dl), hOD = shfl_dn_r(oD, dl);
    if (lane < dl) { lEA = R(0); lEB = R(1); lEC = R(0); lED = R(0); lOA = R(0); lOB = R(1); lOC = R(0); lOD = R(0); }
    if (lane + dl > 31) { hEA = R(0); hEB = R(1); hEC = R(0); hED = R(0); hOA = R(0); hOB = R(1); hOC = R(0); hOD = R(0); }
    {
      const R k1 = eA / lEB, k2 = eC / hEB;
      const R nA = -lEA * k1, nB = eB - lEC * k1 - hEA * k2, nC = -hEC * k2, nD = eD - lED * k1 - hED * k2;
      eA = nA; eB = nB; eC = nC; eD = nD;
    }
    {
      const R k1 = oA / lOB, k2 = oC / hOB;
      const R nA = -lOA * k1, nB = oB - lOC * k1 - hOA * k2, nC = -hOC * k2, nD = oD - lOD * k1 - hOD * k2;
      oA = nA; oB = nB; oC = nC; oD = nD;
    }
  }
  const R x0 = eD / eB;
  const R xl = oD / oB;
  // back-substitution
  d[0] = x0;
  for (int k = 1; k < m - 1; ++k) d[k] = d[k] - a[k] * x0 - c[k] * xl;
  d[m - 1] = xl;
}

}  // namespace ixb
