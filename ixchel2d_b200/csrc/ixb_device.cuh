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

// First statement of every kernel of the SIMPLE loop: wait for the previous
// kernel of the stream (programmatic dependent launch) and let the next one
// be placed.
#define IXB_PDL_ENTRY()                        \
  do {                                         \
    cudaGridDependencySynchronize();           \
    cudaTriggerProgrammaticLaunchCompletion(); \
  } while (0)

// metric arrays inside one device buffer, each `mstride` long, 1-based.
// M_HXU/M_HYV are the energy equation's face diffusivities
// hmean(ge,ge,fexu(k)) / hmean(ge,ge,feyv(k)), M_RHXU/M_RHYV their
// reciprocals (fast form), filled by the table kernel.  The fast form also
// forms the diffusive conductances gamma*delta/d of the 2-D tables below
// from 1-D factors (a uniform gamma makes them separable): M_GRDXP =
// gamma_momen/dxp, M_GRDYV = gamma_momen/dyv, M_GRDXU = gamma_momen/dxu,
// M_GRDYP = gamma_momen/dyp, M_HRDXU = M_HXU/dxu, M_HRDYV = M_HYV/dyv.
enum Metric {
  M_DXP = 0, M_DYP, M_DXU, M_DYU, M_DXV, M_DYV, M_FEXP, M_FEYP, M_FEXU, M_FEYV,
  M_HXU, M_HYV, M_RHXU, M_RHYV, M_GRDXP, M_GRDYV, M_GRDXU, M_GRDYP, M_HRDXU, M_HRDYV, M_COUNT
};

// Mesh-constant 2-D tables (field layout).  With the uniform diffusion
// coefficients of the reference (main.f90:226-239) every harmonic face
// diffusivity and every diffusive conductance gamma*delta/d of the assembly
// is a function of the mesh alone; the table kernel evaluates each one once,
// with the reference's operands in the reference's order, so reading a table
// entry gives the same bits as recomputing it in the cell loop.
//   T_GU (ii,jj)  u: gamman at (ii,jj); gammas(ii,jj) = T_GU(ii,jj-1)
//   T_CU1(ii,jj)  u: gammai*deltay/di;  AD conductance = T_CU1(ii+1,jj)
//   T_CU2(ii,jj)  u: gamman*deltax/dn;  BS conductance = T_CU2(ii,jj-1)
//   T_GV (ii,jj)  v: gammad at (ii,jj); gammai(ii,jj) = T_GV(ii-1,jj)
//   T_CV1(ii,jj)  v: gammai*deltayv/di; AD conductance = T_CV1(ii+1,jj)
//   T_CV2(ii,jj)  v: gammas*deltaxv/ds; BN conductance = T_CV2(ii,jj+1)
//   T_CT1(ii,jj)  T: gammai*deltayp/di; AD conductance = T_CT1(ii+1,jj)
//   T_CT2(ii,jj)  T: gamman*deltaxp/dn; BS conductance = T_CT2(ii,jj-1)
//   (the fast form divides the Peclet numbers of u and v by multiplying with
//   the scalar 1/gamma_momen: the face diffusivities of a uniform gamma)
enum Table { T_GU = 0, T_CU1, T_CU2, T_GV, T_CV1, T_CV2, T_CT1, T_CT2, T_COUNT };

// sweeps: the eight line-solve phases of main.f90
enum Eq { EQ_UY = 0, EQ_UX, EQ_VY, EQ_VX, EQ_PY, EQ_PX, EQ_TY, EQ_TX, EQ_COUNT };

struct BCEntry {  // effective boundary row of one line (last covering segment wins)
  double val;
  int type;       // 0 none, 1 diri, 2 neum
  int pad;
};

struct BatchNorm {          // per-instance norms of a batched launch
  double* partials;         // one per work item of the launch (null: no norm)
  unsigned int* counter;    // one per instance
  double* result;           // one per instance
};

struct NormSlot {        // deterministic two-level sum of squares
  double* partials;      // one per CTA
  unsigned int* counter; // CTAs finished (reset by the last one)
  double* result;        // sqrt(sum) written by the last CTA
};

// Read-only loads of the assembly: every array an assembly reads is left
// untouched by the kernel that reads it, so the non-coherent path applies
// and the compiler may batch the loads ahead of the shared-memory stores.
template <class R>
__device__ __forceinline__ R ldg(const R* p, int i) { return __ldg(p + i); }
// the same load converted to the assembly's arithmetic type (a no-op when
// the field and the arithmetic are both binary64)
template <class R, class F>
__device__ __forceinline__ R ld(const F* p, int i) { return R(__ldg(p + i)); }
template <class R>
struct Geo {
  int mi, nj, LD, mstride;
  int tstride;     // elements per 2-D table (fields stay below 2^31 elements)
  const R* m;      // M_COUNT 1-D arrays
  const R* tab;    // T_COUNT 2-D tables
  R gm, ge, Ri, Riy, dt, rel_vel, rel_pres, rel_ener, p_update;
  R inv_gm, inv_dt, inv_rel_vel, inv_rel_pres, inv_rel_ener;  // fast form
  __device__ __forceinline__ R met(int which, int k) const { return __ldg(m + which * mstride + k); }
  __device__ __forceinline__ int at(int ii, int jj) const { return (jj - 1) * LD + (ii - 1); }
  __device__ __forceinline__ R t(int which, int ii, int jj) const { return __ldg(tab + which * tstride + at(ii, jj)); }
};

// Diffusive conductances of the assembly.  Exact form: the 2-D table entry
// (the reference's operands in its order).  Fast form: the product of the
// cell's 1-D mesh factor, which the caller holds already (`f`), and a 1-D
// reciprocal factor, an L1-resident load in place of a 2-D table read; it
// differs from the table by rounding (the face diffusivities of a uniform
// gamma are gamma itself up to rounding, as in the Peclet numbers).
//   u: T_CU1(ii,jj) = dyu(jj) * GRDXP(ii);   T_CU2(ii,jj) = dxu(ii) * GRDYV(jj)
//   v: T_CV1(ii,jj) = dyv(jj) * GRDXU(ii-1); T_CV2(ii,jj) = dxv(ii) * GRDYP(jj)
//   T: T_CT1(ii,jj) = dyp(jj) * HRDXU(ii-1); T_CT2(ii,jj) = dxp(ii) * HRDYV(jj)
template <bool FAST, class R>
__device__ __forceinline__ R cond_t(const Geo<R>& G, int table, int ii, int jj, R f, int metric, int k) {
  if constexpr (FAST) return f * G.met(metric, k);
  else return G.t(table, ii, jj);
}

template <class R>
struct SweepIO {
  const R *u, *v, *T, *p, *pc;        // current fields
  const R *u_ant, *v_ant, *T_ant;
  const R *au, *av;
  const R *fcon, *flin;               // sources of this equation (null when none)
  const R* in;                        // swept field, current values
  R* out;                             // swept field, new values
  const R* prev;                      // field at the start of the inner pass (null: zero)
  R* aux;                             // au (u-x), av (v-x), b_o (p'-x)
  const BCEntry* bc_first;            // indexed by line
  const BCEntry* bc_last;
  NormSlot nrm0;                      // ||out - prev|| over interior rows of solved lines
  NormSlot nrm1;                      // ||b_o|| (p'-x)
};

template <class R>
struct Row { R a, b, c, d; };

// math on either binary32 or binary64 operands without promotion
__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fabsT(float x) { return fabsf(x); }
__device__ __forceinline__ double fabsT(double x) { return fabs(x); }
__device__ __forceinline__ float fmaxT(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double fmaxT(double a, double b) { return fmax(a, b); }

// DMAX1(0, (1 - 0.1|P|)**5): the integer power as binary powering x*((x*x)*(x*x))
template <class R>
__device__ __forceinline__ R plaw(R pe) {
  R t = R(1) - R(0.1) * fabsT(pe);
  R t2 = t * t;
  R t5 = t * (t2 * t2);
  return fmaxT(R(0), t5);
}
template <class R>
__device__ __forceinline__ R dmax0(R x) { return fmaxT(R(0), x); }

// harmonic face interpolation g1*g2/(g1*(1-f)+g2*f) of the reference
// (e.g. source/mod_ec_momento.f90:462-465) with its operand order
template <class R>
__device__ __forceinline__ R hmean(R g1, R g2, R f) {
  return (g1 * g2) / (g1 * (R(1) - f) + g2 * f);
}

// Reciprocal for the fast form: Newton-Raphson refinement
// r <- r + r(1 - x r) of a hardware reciprocal estimate (two steps for
// binary64, one for binary32).
__device__ __forceinline__ double fast_rcp(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  r = fma(r, fma(-x, r, 1.0), r);
  r = fma(r, fma(-x, r, 1.0), r);
  return r;
}
__device__ __forceinline__ float fast_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return fmaf(r, fmaf(-x, r, 1.0f), r);
}

// a / b.  EXACT (FAST=false): the IEEE quotient of the reference.  FAST:
// a * rb with rb ~ 1/b precomputed (or, when rb is not given, estimated).
template <bool FAST, class R>
__device__ __forceinline__ R qdiv(R a, R b, R rb) { if constexpr (FAST) return a * rb; else return a / b; }
template <bool FAST, class R>
__device__ __forceinline__ R qdiv(R a, R b) { if constexpr (FAST) return a * fast_rcp(b); else return a / b; }

// ---------------------------------------------------------------------------
// u momentum (ensambla_velu_x/_y, source/mod_ec_momento.f90:365-724)
// ---------------------------------------------------------------------------
// The four neighbour coefficients of the u row (:512-526), face velocities
// interpolated as in :447-455, diffusivities and conductances from the
// tables (gammai = gammad = gamma_momen).
template <bool FAST, class R, class F>
__device__ __forceinline__ void u_parts(const Geo<R>& G, const SweepIO<F>& io, const F* u, int ii, int jj,
                                        R& AI, R& AD, R& BS, R& BN, R& deltax, R& deltay, R& temp_int) {
  const F* v = io.v;
  const R fexu_i = G.met(M_FEXU, ii), fexu_m = G.met(M_FEXU, ii - 1);
  const R fexp_i = G.met(M_FEXP, ii);
  R ud = fexu_i * ld<R>(u, G.at(ii + 1, jj)) + (R(1) - fexu_i) * ld<R>(u, G.at(ii, jj));
  R ui = fexu_m * ld<R>(u, G.at(ii, jj)) + (R(1) - fexu_m) * ld<R>(u, G.at(ii - 1, jj));
  R vn = fexp_i * ld<R>(v, G.at(ii + 1, jj)) + (R(1) - fexp_i) * ld<R>(v, G.at(ii, jj));
  R vs = fexp_i * ld<R>(v, G.at(ii + 1, jj - 1)) + (R(1) - fexp_i) * ld<R>(v, G.at(ii, jj - 1));
  const R g = G.gm;
  R gamman, gammas, rgn = R(0), rgs = R(0);
  if constexpr (FAST) {
    // the face diffusivity is the harmonic mean of a uniform gamma_momen
    // (ixb_params holds one value), i.e. gamma_momen up to rounding: its
    // reciprocal is the scalar 1/gamma_momen, no table load
    rgn = rgs = G.inv_gm;
    gamman = gammas = R(0);
  } else {
    gamman = G.t(T_GU, ii, jj);
    gammas = G.t(T_GU, ii, jj - 1);
  }
  R di = G.met(M_DXP, ii), dd = G.met(M_DXP, ii + 1), ds = G.met(M_DYV, jj - 1), dn = G.met(M_DYV, jj);
  deltax = G.met(M_DXU, ii);
  deltay = G.met(M_DYU, jj);
  temp_int = fexp_i * ld<R>(io.T, G.at(ii + 1, jj)) + (R(1) - fexp_i) * ld<R>(io.T, G.at(ii, jj));
  AI = -(cond_t<FAST>(G, T_CU1, ii, jj, deltay, M_GRDXP, ii) * plaw(qdiv<FAST>(ui * di, g, G.inv_gm)) + dmax0(ui * deltay));
  AD = -(cond_t<FAST>(G, T_CU1, ii + 1, jj, deltay, M_GRDXP, ii + 1) * plaw(qdiv<FAST>(ud * dd, g, G.inv_gm)) +
         dmax0(-ud * deltay));
  BS = -(cond_t<FAST>(G, T_CU2, ii, jj - 1, deltax, M_GRDYV, jj - 1) * plaw(qdiv<FAST>(vs * ds, gammas, rgs)) +
         dmax0(vs * deltax));
  BN = -(cond_t<FAST>(G, T_CU2, ii, jj, deltax, M_GRDYV, jj) * plaw(qdiv<FAST>(vn * dn, gamman, rgn)) +
         dmax0(-vn * deltax));
}

// X form (ensambla_velu_x): a=AI c=AD b=AC d=Rx, aux = au = AC*rel
template <bool FAST, class R, class F>
__device__ __forceinline__ Row<R> assemble_ux(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj, R& au) {
  const F* u = io.in;
  R AI, AD, BS, BN, dx, dy, tint;
  u_parts<FAST>(G, io, u, ii, jj, AI, AD, BS, BN, dx, dy, tint);
  const int c0 = G.at(ii, jj);
  const R flin = io.flin ? ld<R>(io.flin, c0) : R(0);  // no sources: no loads (the values would be +0)
  const R fcon = io.fcon ? ld<R>(io.fcon, c0) : R(0);
  Row<R> r;
  r.a = AI;
  r.c = AD;
  r.b = qdiv<FAST>(-AI - AD - BS - BN - dx * dy * flin + qdiv<FAST>(dx * dy, G.dt, G.inv_dt), G.rel_vel,
                   G.inv_rel_vel);
  r.d = -BS * ld<R>(u, G.at(ii, jj - 1)) - BN * ld<R>(u, G.at(ii, jj + 1)) - dx * dy * G.Ri * tint + dx * dy * fcon +
        qdiv<FAST>(dx * dy * ld<R>(io.u_ant, c0), G.dt, G.inv_dt) + (ld<R>(io.p, c0) - ld<R>(io.p, G.at(ii + 1, jj))) * dy +
        r.b * (R(1) - G.rel_vel) * ld<R>(u, c0);
  au = r.b * G.rel_vel;
  return r;
}

// Y form (ensambla_velu_y): a=BS c=BN b=BC d=Ry
template <bool FAST, class R, class F>
__device__ __forceinline__ Row<R> assemble_uy(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj) {
  const F* u = io.in;
  R AI, AD, BS, BN, dx, dy, tint;
  u_parts<FAST>(G, io, u, ii, jj, AI, AD, BS, BN, dx, dy, tint);
  const int c0 = G.at(ii, jj);
  const R flin = io.flin ? ld<R>(io.flin, c0) : R(0);  // no sources: no loads (the values would be +0)
  const R fcon = io.fcon ? ld<R>(io.fcon, c0) : R(0);
  Row<R> r;
  r.a = BS;
  r.c = BN;
  r.b = qdiv<FAST>(-AI - AD - BS - BN - dx * dy * flin + qdiv<FAST>(dx * dy, G.dt, G.inv_dt), G.rel_vel,
                   G.inv_rel_vel);
  r.d = -AI * ld<R>(u, G.at(ii - 1, jj)) - AD * ld<R>(u, G.at(ii + 1, jj)) - dx * dy * G.Ri * tint + dx * dy * fcon +
        qdiv<FAST>(dx * dy * ld<R>(io.u_ant, c0), G.dt, G.inv_dt) + (ld<R>(io.p, c0) - ld<R>(io.p, G.at(ii + 1, jj))) * dy +
        r.b * (R(1) - G.rel_vel) * ld<R>(u, c0);
  return r;
}

// ---------------------------------------------------------------------------
// v momentum (ensambla_velv_x/_y, source/mod_ec_momento.f90:736-1098)
// ---------------------------------------------------------------------------
template <bool FAST, class R, class F>
__device__ __forceinline__ void v_parts(const Geo<R>& G, const SweepIO<F>& io, const F* v, int ii, int jj,
                                        R& AI, R& AD, R& BS, R& BN, R& temp_int) {
  const F* u = io.u;
  const R feyp_j = G.met(M_FEYP, jj);
  const R feyv_j = G.met(M_FEYV, jj), feyv_m = G.met(M_FEYV, jj - 1);
  R ud = feyp_j * ld<R>(u, G.at(ii, jj + 1)) + (R(1) - feyp_j) * ld<R>(u, G.at(ii, jj));
  R ui = feyp_j * ld<R>(u, G.at(ii - 1, jj + 1)) + (R(1) - feyp_j) * ld<R>(u, G.at(ii - 1, jj));
  R vn = feyv_j * ld<R>(v, G.at(ii, jj + 1)) + (R(1) - feyv_j) * ld<R>(v, G.at(ii, jj));
  R vs = feyv_m * ld<R>(v, G.at(ii, jj)) + (R(1) - feyv_m) * ld<R>(v, G.at(ii, jj - 1));
  const R g = G.gm;  // gamman = gammas = gamma_momen (:854-858)
  R gammad, gammai, rgd = R(0), rgi = R(0);
  if constexpr (FAST) {
    rgd = rgi = G.inv_gm;  // uniform gamma_momen, as in u_parts
    gammad = gammai = R(0);
  } else {
    gammad = G.t(T_GV, ii, jj);
    gammai = G.t(T_GV, ii - 1, jj);
  }
  R di = G.met(M_DXU, ii - 1), dd = G.met(M_DXU, ii), ds = G.met(M_DYP, jj), dn = G.met(M_DYP, jj + 1);
  const R dyv = G.met(M_DYV, jj), dxv = G.met(M_DXV, ii);
  temp_int = feyp_j * ld<R>(io.T, G.at(ii, jj + 1)) + (R(1) - feyp_j) * ld<R>(io.T, G.at(ii, jj));
  AI = -(cond_t<FAST>(G, T_CV1, ii, jj, dyv, M_GRDXU, ii - 1) * plaw(qdiv<FAST>(ui * di, gammai, rgi)) +
         dmax0(ui * dyv));
  AD = -(cond_t<FAST>(G, T_CV1, ii + 1, jj, dyv, M_GRDXU, ii) * plaw(qdiv<FAST>(ud * dd, gammad, rgd)) +
         dmax0(-ud * dyv));
  BS = -(cond_t<FAST>(G, T_CV2, ii, jj, dxv, M_GRDYP, jj) * plaw(qdiv<FAST>(vs * ds, g, G.inv_gm)) + dmax0(vs * dxv));
  BN = -(cond_t<FAST>(G, T_CV2, ii, jj + 1, dxv, M_GRDYP, jj + 1) * plaw(qdiv<FAST>(vn * dn, g, G.inv_gm)) +
         dmax0(-vn * dxv));
}

template <bool FAST, class R, class F>
__device__ __forceinline__ Row<R> assemble_vx(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj, R& av) {
  const F* v = io.in;
  R AI, AD, BS, BN, tint;
  v_parts<FAST>(G, io, v, ii, jj, AI, AD, BS, BN, tint);
  const int c0 = G.at(ii, jj);
  const R dxv = G.met(M_DXV, ii), dyv = G.met(M_DYV, jj);
  const R dxdy = dxv * dyv;
  const R flin = io.flin ? ld<R>(io.flin, c0) : R(0);  // no sources: no loads (the values would be +0)
  const R fcon = io.fcon ? ld<R>(io.fcon, c0) : R(0);
  Row<R> r;
  r.a = AI;
  r.c = AD;
  r.b = qdiv<FAST>(-AI - AD - BS - BN - dxdy * flin + qdiv<FAST>(dxdy, G.dt, G.inv_dt), G.rel_vel, G.inv_rel_vel);
  r.d = -BS * ld<R>(v, G.at(ii, jj - 1)) - BN * ld<R>(v, G.at(ii, jj + 1)) - dxdy * G.Riy * tint + dxdy * fcon +
        qdiv<FAST>(dxdy * ld<R>(io.v_ant, c0), G.dt, G.inv_dt) + (ld<R>(io.p, c0) - ld<R>(io.p, G.at(ii, jj + 1))) * dxv +
        r.b * (R(1) - G.rel_vel) * ld<R>(v, c0);
  av = r.b * G.rel_vel;
  return r;
}

template <bool FAST, class R, class F>
__device__ __forceinline__ Row<R> assemble_vy(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj) {
  const F* v = io.in;
  R AI, AD, BS, BN, tint;
  v_parts<FAST>(G, io, v, ii, jj, AI, AD, BS, BN, tint);
  const int c0 = G.at(ii, jj);
  const R dxv = G.met(M_DXV, ii), dyv = G.met(M_DYV, jj);
  const R dxdy = dxv * dyv;
  const R flin = io.flin ? ld<R>(io.flin, c0) : R(0);  // no sources: no loads (the values would be +0)
  const R fcon = io.fcon ? ld<R>(io.fcon, c0) : R(0);
  Row<R> r;
  r.a = BS;
  r.c = BN;
  r.b = qdiv<FAST>(-AI - AD - BS - BN - dxdy * flin + qdiv<FAST>(dxdy, G.dt, G.inv_dt), G.rel_vel, G.inv_rel_vel);
  r.d = -AI * ld<R>(v, G.at(ii - 1, jj)) - AD * ld<R>(v, G.at(ii + 1, jj)) - dxdy * G.Riy * tint + dxdy * fcon +
        qdiv<FAST>(dxdy * ld<R>(io.v_ant, c0), G.dt, G.inv_dt) + (ld<R>(io.p, c0) - ld<R>(io.p, G.at(ii, jj + 1))) * dxv +
        r.b * (R(1) - G.rel_vel) * ld<R>(v, c0);
  return r;
}

// ---------------------------------------------------------------------------
// energy (ensambla_energia_x/_y, source/mod_ec_energia.f90:119-443).  The
// calls in main.f90:989 and :1060 bind fexu/feyv to the dummies fexpo/feypo.
// ---------------------------------------------------------------------------
template <bool FAST, class R, class F>
__device__ __forceinline__ void t_parts(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj, R& AI, R& AD,
                                        R& BS, R& BN) {
  const R ud = ld<R>(io.u, G.at(ii, jj)), ui = ld<R>(io.u, G.at(ii - 1, jj));
  const R vn = ld<R>(io.v, G.at(ii, jj)), vs = ld<R>(io.v, G.at(ii, jj - 1));
  const R di = G.met(M_DXU, ii - 1), dd = G.met(M_DXU, ii), ds = G.met(M_DYV, jj - 1), dn = G.met(M_DYV, jj);
  const R dyp = G.met(M_DYP, jj), dxp = G.met(M_DXP, ii);
  if constexpr (FAST) {
    AI = -(cond_t<true>(G, T_CT1, ii, jj, dyp, M_HRDXU, ii - 1) * plaw(ui * di * G.met(M_RHXU, ii - 1)) +
           dmax0(ui * dyp));
    AD = -(cond_t<true>(G, T_CT1, ii + 1, jj, dyp, M_HRDXU, ii) * plaw(ud * dd * G.met(M_RHXU, ii)) + dmax0(-ud * dyp));
    BS = -(cond_t<true>(G, T_CT2, ii, jj - 1, dxp, M_HRDYV, jj - 1) * plaw(vs * ds * G.met(M_RHYV, jj - 1)) +
           dmax0(vs * dxp));
    BN = -(cond_t<true>(G, T_CT2, ii, jj, dxp, M_HRDYV, jj) * plaw(vn * dn * G.met(M_RHYV, jj)) + dmax0(-vn * dxp));
  } else {
    const R gammad = G.met(M_HXU, ii);
    const R gammai = G.met(M_HXU, ii - 1);
    const R gamman = G.met(M_HYV, jj);
    const R gammas = G.met(M_HYV, jj - 1);
    AI = -(G.t(T_CT1, ii, jj) * plaw(ui * di / gammai) + dmax0(ui * dyp));
    AD = -(G.t(T_CT1, ii + 1, jj) * plaw(ud * dd / gammad) + dmax0(-ud * dyp));
    BS = -(G.t(T_CT2, ii, jj - 1) * plaw(vs * ds / gammas) + dmax0(vs * dxp));
    BN = -(G.t(T_CT2, ii, jj) * plaw(vn * dn / gamman) + dmax0(-vn * dxp));
  }
}

template <bool FAST, class R, class F>
__device__ __forceinline__ Row<R> assemble_tx(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj) {
  const F* T = io.in;
  R AI, AD, BS, BN;
  t_parts<FAST>(G, io, ii, jj, AI, AD, BS, BN);
  const int c0 = G.at(ii, jj);
  const R dxdy = G.met(M_DXP, ii) * G.met(M_DYP, jj);
  const R flin = io.flin ? ld<R>(io.flin, c0) : R(0);  // no sources: no loads (the values would be +0)
  const R fcon = io.fcon ? ld<R>(io.fcon, c0) : R(0);
  Row<R> r;
  r.a = AI;
  r.c = AD;
  r.b = qdiv<FAST>(-AI - AD - BS - BN - dxdy * flin + qdiv<FAST>(dxdy, G.dt, G.inv_dt), G.rel_ener, G.inv_rel_ener);
  r.d = -BS * ld<R>(T, G.at(ii, jj - 1)) - BN * ld<R>(T, G.at(ii, jj + 1)) + dxdy * fcon +
        qdiv<FAST>(dxdy * ld<R>(io.T_ant, c0), G.dt, G.inv_dt) + r.b * (R(1) - G.rel_ener) * ld<R>(T, c0);
  return r;
}

template <bool FAST, class R, class F>
__device__ __forceinline__ Row<R> assemble_ty(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj) {
  const F* T = io.in;
  R AI, AD, BS, BN;
  t_parts<FAST>(G, io, ii, jj, AI, AD, BS, BN);
  const int c0 = G.at(ii, jj);
  const R dxdy = G.met(M_DXP, ii) * G.met(M_DYP, jj);
  const R flin = io.flin ? ld<R>(io.flin, c0) : R(0);  // no sources: no loads (the values would be +0)
  const R fcon = io.fcon ? ld<R>(io.fcon, c0) : R(0);
  Row<R> r;
  r.a = BS;
  r.c = BN;
  r.b = qdiv<FAST>(-AI - AD - BS - BN - dxdy * flin + qdiv<FAST>(dxdy, G.dt, G.inv_dt), G.rel_ener, G.inv_rel_ener);
  r.d = -AI * ld<R>(T, G.at(ii - 1, jj)) - AD * ld<R>(T, G.at(ii + 1, jj)) + dxdy * fcon +
        qdiv<FAST>(dxdy * ld<R>(io.T_ant, c0), G.dt, G.inv_dt) + r.b * (R(1) - G.rel_ener) * ld<R>(T, c0);
  return r;
}

// ---------------------------------------------------------------------------
// pressure correction (ensambla_corr_pres_x/_y, source/mod_ec_momento.f90:145-355)
// ---------------------------------------------------------------------------
template <class R, class F>
__device__ __forceinline__ R pc_at(const SweepIO<F>& io, const Geo<R>& G, int ii, int jj) {
  return ld<R>(io.in, G.at(ii, jj));
}

// Mass source b_o = (u_w - u_e) dy + (v_s - v_n) dx of the p' rows, always
// in the fields' precision (binary64) with binary64 metrics, whatever the
// precision of the coefficients.
template <class R, class F>
__device__ __forceinline__ F mass_residual(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj) {
  const int c0 = G.at(ii, jj);
  const F ud = ldg(io.u, c0), ui = ldg(io.u, G.at(ii - 1, jj)), vn = ldg(io.v, c0), vs = ldg(io.v, G.at(ii, jj - 1));
  return (ui - ud) * F(G.met(M_DYP, jj)) + (vs - vn) * F(G.met(M_DXP, ii));
}

template <bool FAST, class R, class F>
__device__ __forceinline__ Row<R> assemble_px(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj, F& bo) {
  const int c0 = G.at(ii, jj);
  const R ai = ld<R>(io.au, G.at(ii - 1, jj)), ad = ld<R>(io.au, c0), as = ld<R>(io.av, G.at(ii, jj - 1)),
          an = ld<R>(io.av, c0);
  const R dyp = G.met(M_DYP, jj), dxp = G.met(M_DXP, ii);
  Row<R> r;
  r.a = -qdiv<FAST>(dyp * dyp, ai);
  r.c = -qdiv<FAST>(dyp * dyp, ad);
  const R BS = -qdiv<FAST>(dxp * dxp, as);
  const R BN = -qdiv<FAST>(dxp * dxp, an);
  r.b = qdiv<FAST>(-r.a - r.c - BS - BN, G.rel_pres, G.inv_rel_pres);
  bo = mass_residual(G, io, ii, jj);
  r.d = -BS * pc_at<R>(io, G, ii, jj - 1) - BN * pc_at<R>(io, G, ii, jj + 1) + R(bo) +
        (R(1) - G.rel_pres) * r.b * pc_at<R>(io, G, ii, jj);
  return r;
}

template <bool FAST, class R, class F>
__device__ __forceinline__ Row<R> assemble_py(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj) {
  const int c0 = G.at(ii, jj);
  const R ai = ld<R>(io.au, G.at(ii - 1, jj)), ad = ld<R>(io.au, c0), as = ld<R>(io.av, G.at(ii, jj - 1)),
          an = ld<R>(io.av, c0);
  const R dyp = G.met(M_DYP, jj), dxp = G.met(M_DXP, ii);
  const R AI = -qdiv<FAST>(dyp * dyp, ai);
  const R AD = -qdiv<FAST>(dyp * dyp, ad);
  Row<R> r;
  r.a = -qdiv<FAST>(dxp * dxp, as);
  r.c = -qdiv<FAST>(dxp * dxp, an);
  r.b = qdiv<FAST>(-AI - AD - r.a - r.c, G.rel_pres, G.inv_rel_pres);
  const R bo = R(mass_residual(G, io, ii, jj));
  r.d = -AI * pc_at<R>(io, G, ii - 1, jj) - AD * pc_at<R>(io, G, ii + 1, jj) + bo +
        (R(1) - G.rel_pres) * r.b * pc_at<R>(io, G, ii, jj);
  return r;
}

// ---------------------------------------------------------------------------
// u residual (residuo_u, source/mod_ec_momento.f90:1107-1266).  With a
// uniform gamma the reference's different south numerator (:1208) has the
// same value as in ensambla_velu_x, so it shares the u tables.
// ---------------------------------------------------------------------------
// T_WRITTEN: T was written earlier in the calling kernel (a fused T-x sweep
// evaluating the residual of the rows it solved), so it is read with
// ordinary coherent loads instead of the read-only path.
template <bool FAST, class R, bool T_WRITTEN = false>
__device__ __forceinline__ R residual_u(const Geo<R>& G, const R* u, const R* v, const R* T, const R* p,
                                        const R* u_ant, const R* fcon, const R* flin, int ii, int jj) {
  const R fexu_i = G.met(M_FEXU, ii), fexu_m = G.met(M_FEXU, ii - 1);
  const R fexp_i = G.met(M_FEXP, ii);
  R ud = fexu_i * ldg(u, G.at(ii + 1, jj)) + (R(1) - fexu_i) * ldg(u, G.at(ii, jj));
  R ui = fexu_m * ldg(u, G.at(ii, jj)) + (R(1) - fexu_m) * ldg(u, G.at(ii - 1, jj));
  R vn = fexp_i * ldg(v, G.at(ii + 1, jj)) + (R(1) - fexp_i) * ldg(v, G.at(ii, jj));
  R vs = fexp_i * ldg(v, G.at(ii + 1, jj - 1)) + (R(1) - fexp_i) * ldg(v, G.at(ii, jj - 1));
  const R g = G.gm;
  R gamman, gammas, rgn = R(0), rgs = R(0);
  if constexpr (FAST) {
    // the face diffusivity is the harmonic mean of a uniform gamma_momen
    // (ixb_params holds one value), i.e. gamma_momen up to rounding: its
    // reciprocal is the scalar 1/gamma_momen, no table load
    rgn = rgs = G.inv_gm;
    gamman = gammas = R(0);
  } else {
    gamman = G.t(T_GU, ii, jj);
    gammas = G.t(T_GU, ii, jj - 1);
  }
  R di = G.met(M_DXP, ii), dd = G.met(M_DXP, ii + 1), ds = G.met(M_DYV, jj - 1), dn = G.met(M_DYV, jj);
  const R dxu = G.met(M_DXU, ii), dyu = G.met(M_DYU, jj);
  const int c0 = G.at(ii, jj);
  const R t_e = T_WRITTEN ? T[G.at(ii + 1, jj)] : ldg(T, G.at(ii + 1, jj));
  const R t_c = T_WRITTEN ? T[c0] : ldg(T, c0);
  R temp_int = fexp_i * t_e + (R(1) - fexp_i) * t_c;
  R AI = (cond_t<FAST>(G, T_CU1, ii, jj, dyu, M_GRDXP, ii) * plaw(qdiv<FAST>(ui * di, g, G.inv_gm)) + dmax0(ui * dyu));
  R AD = (cond_t<FAST>(G, T_CU1, ii + 1, jj, dyu, M_GRDXP, ii + 1) * plaw(qdiv<FAST>(ud * dd, g, G.inv_gm)) +
          dmax0(-ud * dyu));
  R BS = (cond_t<FAST>(G, T_CU2, ii, jj - 1, dxu, M_GRDYV, jj - 1) * plaw(qdiv<FAST>(vs * ds, gammas, rgs)) +
          dmax0(vs * dxu));
  R BN = (cond_t<FAST>(G, T_CU2, ii, jj, dxu, M_GRDYV, jj) * plaw(qdiv<FAST>(vn * dn, gamman, rgn)) +
          dmax0(-vn * dxu));
  const R fl = flin ? ldg(flin, c0) : R(0);
  const R fc = fcon ? ldg(fcon, c0) : R(0);
  R AC = AI + AD + BS + BN - dxu * dyu * fl + qdiv<FAST>(dxu * dyu, G.dt, G.inv_dt);
  return AI * ldg(u, G.at(ii - 1, jj)) - AC * ldg(u, c0) + AD * ldg(u, G.at(ii + 1, jj)) +
         BS * ldg(u, G.at(ii, jj - 1)) + BN * ldg(u, G.at(ii, jj + 1)) - dxu * dyu * G.Ri * temp_int +
         dxu * dyu * fc + qdiv<FAST>(dxu * dyu * ldg(u_ant, c0), G.dt, G.inv_dt) +
         (ldg(p, c0) - ldg(p, G.at(ii + 1, jj))) * dyu;
}

// ---------------------------------------------------------------------------
// Line solvers on a line staged in shared memory.
// Row r of the (padded) line lives in chunk r / m at slot r % m; each row
// array is [G][mp] with mp odd, so G threads walking their chunks in step
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

// Reduced-system solvers of the partitioned line solve
enum ReducedSolve { RS_PCR = 0, RS_WARP = 1 };

__host__ __device__ constexpr int warp_chunk(int G) { return (2 * G + 31) / 32 < 3 ? 3 : (2 * G + 31) / 32; }

// Shared-memory footprint (elements) of one line: the four row arrays of G
// chunks (pitch mp), plus the reduced system: for RS_PCR two buffers of the
// 2G normalised rows (a, c, d), for RS_WARP four [32][m2|1] arrays; room
// for the larger of the two.
__host__ __device__ constexpr size_t line_smem_elems(int G, int mp) {
  return (size_t)4 * G * mp +
         ((size_t)12 * G > (size_t)4 * 32 * (warp_chunk(G) | 1) ? (size_t)12 * G : (size_t)4 * 32 * (warp_chunk(G) | 1));
}

template <class R>
__device__ __forceinline__ R shfl_up_r(R x, int d) { return __shfl_up_sync(0xffffffffu, x, d); }
template <class R>
__device__ __forceinline__ R shfl_dn_r(R x, int d) { return __shfl_down_sync(0xffffffffu, x, d); }

// One warp solves one system staged as [32][mp] chunks of m >= 3 rows:
// every lane eliminates its chunk down to two rows coupled to the
// neighbouring chunks (forward and backward "modified Thomas" sweeps), the
// warp solves the 64-row reduced system by parallel cyclic reduction with
// register shuffles, and every lane back-substitutes its chunk.  (Thomas-PCR
// hybrid of Laszlo, Giles and Appleyard, ACM TOMS 42(4) 2016.)  Must be
// called by all 32 lanes.
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


// Reduced system of a partitioned line solve: the first and last rows of G
// chunks, each with unit diagonal, coupled to the neighbouring chunks' end
// rows (row 2k: eA x_{2k-1} + x_{2k} + eC x_{2k+1} = eD; row 2k+1 likewise
// with oA, oC, oD).  Solved by parallel cyclic reduction over log2(2G) steps
// in shared memory `red` (12 G elements, two buffers of a | c | d); thread
// k supplies rows 2k, 2k+1 and receives their solutions x0, xl.  Called by
// all threads of the CTA (it holds barriers); `active` false: barriers only.
// Barrier of the G threads that solve one line when a CTA holds TL lines of
// whole warps (a named barrier per line, so lines do not wait for each
// other), else of the whole CTA.
template <int G, int TL>
__device__ __forceinline__ void line_sync() {
  if constexpr (TL > 1 && TL <= 8 && G % 32 == 0) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)threadIdx.x / G), "r"(G) : "memory");
  } else {
    __syncthreads();
  }
}

template <class R, int G, int TL = 1>
__device__ __forceinline__ void reduced_pcr(R* red, int k, bool active, R eA, R eC, R eD, R oA, R oC, R oD, R& x0,
                                            R& xl) {
  R* cur = red;
  R* nxt = red + 6 * G;
  if (active) {
    cur[2 * k] = eA; cur[2 * G + 2 * k] = eC; cur[4 * G + 2 * k] = eD;
    cur[2 * k + 1] = oA; cur[2 * G + 2 * k + 1] = oC; cur[4 * G + 2 * k + 1] = oD;
  }
  line_sync<G, TL>();
#pragma unroll 1
  for (int s = 1; s < 2 * G; s <<= 1) {
    if (active) {
      const R* Ac = cur; const R* Cc = cur + 2 * G; const R* Dc = cur + 4 * G;
      R* An = nxt; R* Cn = nxt + 2 * G; R* Dn = nxt + 4 * G;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int i = k + q * G;
        const R ai = Ac[i], ci = Cc[i], di = Dc[i];
        R alo = R(0), clo = R(0), dlo = R(0), ahi = R(0), chi = R(0), dhi = R(0);
        if (i - s >= 0) { alo = Ac[i - s]; clo = Cc[i - s]; dlo = Dc[i - s]; }
        if (i + s < 2 * G) { ahi = Ac[i + s]; chi = Cc[i + s]; dhi = Dc[i + s]; }
        const R r = fast_rcp(fmaT(-ci, ahi, fmaT(-ai, clo, R(1))));
        An[i] = -ai * alo * r;
        Cn[i] = -ci * chi * r;
        Dn[i] = fmaT(-ci, dhi, fmaT(-ai, dlo, di)) * r;
      }
    }
    line_sync<G, TL>();
    R* t = cur; cur = nxt; nxt = t;
  }
  x0 = cur[4 * G + 2 * k];
  xl = cur[4 * G + 2 * k + 1];
}

// Partitioned line solve of the TL lines staged in shared memory, G threads
// per line (thread t: line t / G, chunk k = t % G, rows k*m .. k*m+m-1 at
// offset k*mp of the line's row arrays).  Every thread eliminates its chunk
// (m >= 3 rows) down to two rows coupled only to the neighbouring chunks'
// end rows (a forward and a backward "modified Thomas" sweep); the 2G
// reduced rows of each line are then solved either by parallel cyclic
// reduction over all G threads in shared memory (RS_PCR, log2(2G) steps) or
// by one warp per line with the warp Thomas-PCR hybrid (RS_WARP); finally
// every thread back-substitutes its chunk.  This is the Thomas-PCR hybrid of
// Laszlo, Giles and Appleyard (ACM TOMS 42(4), 2016) applied twice.
// Reciprocals use fast_rcp (two Newton steps).  The solution replaces the
// right-hand side.  Called by all TL*G threads;
// threads of lines with `active` false only take part in the barriers.
template <class R, int G, int TL = 1>
__device__ __forceinline__ void chunk_solve(R* line, int m, int mp, bool active, int rs) {
  const int k = threadIdx.x % G;
  R* a = line + k * mp;
  R* b = a + (size_t)G * mp;
  R* c = b + (size_t)G * mp;
  R* d = c + (size_t)G * mp;
  R* red = line + (size_t)4 * G * mp;
  constexpr int M2 = warp_chunk(G);
  constexpr int M2P = M2 | 1;
  R eA = R(0), eC = R(0), eD = R(0), oA = R(0), oC = R(0), oD = R(0);
  if (active) {
    // forward: rows 1..m-1 -> x_k + a'_k x_0 + c'_k x_{k+1} = d'_k
    const R a0 = a[0], b0 = b[0], c0 = c[0], d0 = d[0];
    R inv = fast_rcp(b[1]);
    R ap = a[1] * inv, cp = c[1] * inv, dp = d[1] * inv;
    a[1] = ap; c[1] = cp; d[1] = dp;
    for (int i = 2; i < m; ++i) {
      const R ai = a[i];
      const R r = fast_rcp(fmaT(-ai, cp, b[i]));
      ap = -ai * ap * r;
      dp = fmaT(-ai, dp, d[i]) * r;
      cp = c[i] * r;
      a[i] = ap; c[i] = cp; d[i] = dp;
    }
    // backward: rows m-3..1 -> x_i + a''_i x_0 + c''_i x_{m-1} = d''_i
    R an = a[m - 2], cn = c[m - 2], dn = d[m - 2];
    for (int i = m - 3; i >= 1; --i) {
      const R ci = c[i];
      dn = fmaT(-ci, dn, d[i]);
      an = fmaT(-ci, an, a[i]);
      cn = -ci * cn;
      a[i] = an; c[i] = cn; d[i] = dn;
    }
    // reduced rows 2k (chunk's first row) and 2k+1 (its last row), unit diagonal
    const R r0 = fast_rcp(fmaT(-c0, an, b0));
    eA = a0 * r0; eC = -c0 * cn * r0; eD = fmaT(-c0, dn, d0) * r0;
    oA = ap; oC = cp; oD = dp;
  }
  R x0, xl;
  if (rs == RS_PCR) {
    reduced_pcr<R, G, TL>(red, k, active, eA, eC, eD, oA, oC, oD, x0, xl);
  } else {
    // reduced system in the warp solver's [32][M2P] chunk layout
    constexpr int ARR2 = 32 * M2P;
    auto off = [](int q) { return (q / M2) * M2P + q % M2; };
    if (active) {
      int o = off(2 * k);
      red[o] = eA; red[o + ARR2] = R(1); red[o + 2 * ARR2] = eC; red[o + 3 * ARR2] = eD;
      o = off(2 * k + 1);
      red[o] = oA; red[o + ARR2] = R(1); red[o + 2 * ARR2] = oC; red[o + 3 * ARR2] = oD;
    }
    // identity rows pad the reduced system to 32*M2 rows
    for (int q = 2 * G + k; q < 32 * M2; q += G) {
      const int o = off(q);
      red[o] = R(0); red[o + ARR2] = R(1); red[o + 2 * ARR2] = R(0); red[o + 3 * ARR2] = R(0);
    }
    __syncthreads();
    if (k < 32 && active) thomas_pcr_warp(red, red + ARR2, red + 2 * ARR2, red + 3 * ARR2, M2, M2P);
    __syncthreads();
    x0 = red[3 * ARR2 + off(2 * k)];
    xl = red[3 * ARR2 + off(2 * k + 1)];
  }
  if (active) {
    d[0] = x0;
    for (int i = 1; i < m - 1; ++i) d[i] = fmaT(-c[i], xl, fmaT(-a[i], x0, d[i]));
    d[m - 1] = xl;
  }
}

}  // namespace ixb
