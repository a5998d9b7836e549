// ixb_kernels.cu -- the non-sweep kernels of the SIMPLE outer iteration
// (p/u/v correction, u residual, Nusselt number, mesh-constant tables), the
// launch shape of the sweeps and their dispatch to the per-equation
// translation units.
#include <mutex>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "ixb_ctl.cuh"
#include "ixb_nusselt.h"
#include "ixb_internal.h"
#include "ixb_reduce.cuh"

namespace ixb {

// ---------------------------------------------------------------------------
// mesh-constant tables (see ixb_device.cuh), one thread per (ii,jj);
// operands in the reference's order (-fmad=false build)
// ---------------------------------------------------------------------------
template <class R>
__global__ void table1d_kernel(Geo<R> G, R* met) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const R ge = G.ge;
  // 1-D factor num / d of the fast form's conductances (0 where d is not set)
  auto ratio = [](R num, R d) { return d != R(0) ? num / d : R(0); };
  const R g = G.gm;
  if (k >= 1 && k <= G.mi) {
    const R h = hmean(ge, ge, G.met(M_FEXU, k));
    met[M_HXU * G.mstride + k] = h;
    met[M_RHXU * G.mstride + k] = R(1) / h;
    met[M_HRDXU * G.mstride + k] = ratio(h, G.met(M_DXU, k));
  }
  if (k >= 1 && k <= G.nj) {
    const R h = hmean(ge, ge, G.met(M_FEYV, k));
    met[M_HYV * G.mstride + k] = h;
    met[M_RHYV * G.mstride + k] = R(1) / h;
    met[M_HRDYV * G.mstride + k] = ratio(h, G.met(M_DYV, k));
  }
  if (k >= 1 && k < G.mstride) {
    met[M_GRDXP * G.mstride + k] = ratio(g, G.met(M_DXP, k));
    met[M_GRDYV * G.mstride + k] = ratio(g, G.met(M_DYV, k));
    met[M_GRDXU * G.mstride + k] = ratio(g, G.met(M_DXU, k));
    met[M_GRDYP * G.mstride + k] = ratio(g, G.met(M_DYP, k));
  }
}

template <class R>
__global__ void table2d_kernel(Geo<R> G, R* tab) {
  const int ii = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int jj = 1 + blockIdx.y;
  if (ii > G.mi + 1 || jj > G.nj + 1) return;
  const size_t c0 = G.at(ii, jj);
  auto T = [&](int w) -> R& { return tab[w * G.tstride + c0]; };
  const R g = G.gm;
  auto combo = [](R h, R f) { return h * h / (h * (R(1) - f) + h * f); };
  // u (ensambla_velu_x :462-479, :512-526)
  if (ii <= G.mi && jj <= G.nj) {
    const R hy = hmean(g, g, G.met(M_FEYP, jj));
    const R gamman = combo(hy, G.met(M_FEXP, ii));
    T(T_GU) = gamman;
    T(T_CU2) = gamman * G.met(M_DXU, ii) / G.met(M_DYV, jj);
  }
  if (ii >= 2 && ii <= G.mi && jj >= 2 && jj <= G.nj) T(T_CU1) = g * G.met(M_DYU, jj) / G.met(M_DXP, ii);
  // v (ensambla_velv_x :833-850, :880-894)
  if (ii <= G.mi && jj <= G.nj) {
    const R hx = hmean(g, g, G.met(M_FEXP, ii));
    T(T_GV) = combo(hx, G.met(M_FEYP, jj));
  }
  if (ii >= 2 && ii <= G.mi + 1 && jj <= G.nj) {
    const R hx = hmean(g, g, G.met(M_FEXP, ii - 1));
    const R gammai = combo(hx, G.met(M_FEYP, jj));
    T(T_CV1) = gammai * G.met(M_DYV, jj) / G.met(M_DXU, ii - 1);
  }
  if (ii >= 2 && ii <= G.mi && jj >= 2 && jj <= G.nj) T(T_CV2) = g * G.met(M_DXV, ii) / G.met(M_DYP, jj);
  // T (ensambla_energia_x :230-259, fexu/feyv bound to fexpo/feypo)
  const R ge = G.ge;
  if (ii >= 2 && ii <= G.mi + 1 && jj >= 2 && jj <= G.nj) {
    const R gammai = hmean(ge, ge, G.met(M_FEXU, ii - 1));
    T(T_CT1) = gammai * G.met(M_DYP, jj) / G.met(M_DXU, ii - 1);
  }
  if (ii >= 2 && ii <= G.mi && jj <= G.nj) {
    const R gamman = hmean(ge, ge, G.met(M_FEYV, jj));
    T(T_CT2) = gamman * G.met(M_DXP, ii) / G.met(M_DYV, jj);
  }
}

cudaError_t launch_tables_f64(const Geo<double>& G, double* met, double* tab, cudaStream_t st) {
  const int n1 = std::max(G.mi, G.nj) + 1;
  table1d_kernel<double><<<(n1 + 127) / 128, 128, 0, st>>>(G, met);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dim3 grid((G.mi + 1 + 127) / 128, G.nj + 1);
  table2d_kernel<double><<<grid, 128, 0, st>>>(G, tab);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// pressure and velocity correction, main.f90:931-962
// ---------------------------------------------------------------------------
template <class R, bool FAST>
__device__ __forceinline__ void correct_cell(const Geo<R>& G, R* __restrict__ u, R* __restrict__ v, R* __restrict__ p,
                                             const R* __restrict__ pc, const R* __restrict__ au,
                                             const R* __restrict__ av, int idx) {
  const int ni = G.mi - 1;  // ii = 2..mi
  const int ii = 2 + idx % ni;
  const int jj = 2 + idx / ni;
  const size_t c0 = G.at(ii, jj);
  // Every load first, then the stores: u at ii = mi and v at jj = nj are
  // boundary values the update leaves alone, but their entries (and those of
  // au, av and p' one cell further) exist, so the three updates' loads go out
  // together instead of one branch after another; the unused results are
  // dropped.
  const R p0 = p[c0], pc0 = pc[c0], pce = pc[G.at(ii + 1, jj)], pcn = pc[G.at(ii, jj + 1)];
  const R u0 = u[c0], au0 = au[c0], v0 = v[c0], av0 = av[c0];
  const R dyu = G.met(M_DYU, jj), dxv = G.met(M_DXV, ii);
  p[c0] = p0 + G.p_update * pc0;
  if (ii <= G.mi - 1) u[c0] = u0 + qdiv<FAST>(dyu * (pc0 - pce), au0);
  if (jj <= G.nj - 1) v[c0] = v0 + qdiv<FAST>(dxv * (pc0 - pcn), av0);
}

template <class R, bool FAST>
__global__ void correct_kernel(const Geo<R> G, R* __restrict__ u, R* __restrict__ v, R* __restrict__ p,
                               const R* __restrict__ pc, const R* __restrict__ au, const R* __restrict__ av,
                               const CtlRef gate) {
  IXB_PDL_ENTRY();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < (G.mi - 1) * (G.nj - 1)) correct_cell<R, FAST>(G, u, v, p, pc, au, av, idx);
  if (gate.ctl && idx == 0) ctl_gate_step(gate.ctl, gate.cond);  // opens the energy loop
}

// p' reset at the start of the pressure loop (main.f90:752-758), opening it
__global__ void preset_kernel(double* __restrict__ pc, size_t n, const CtlRef gate) {
  IXB_PDL_ENTRY();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    pc[i] = 0.0;
  if (gate.ctl && blockIdx.x == 0 && threadIdx.x == 0) ctl_gate_step(gate.ctl, gate.cond);
}

// ---------------------------------------------------------------------------
// u residual and its norm, main.f90:1169-1199
// ---------------------------------------------------------------------------
template <class R, bool FAST>
__global__ void __launch_bounds__(256) residual_kernel(const Geo<R> G, const R* __restrict__ u,
                                                       const R* __restrict__ v, const R* __restrict__ T,
                                                       const R* __restrict__ p, const R* __restrict__ u_ant,
                                                       const R* __restrict__ fcon, const R* __restrict__ flin,
                                                       R* __restrict__ resu, NormSlot ns, const CtlRef outer) {
  IXB_PDL_ENTRY();
  const int ni = G.mi - 2;  // ii = 2..mi-1
  const int total = ni * (G.nj - 1);
  double acc = 0.0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int ii = 2 + idx % ni;
    const int jj = 2 + idx / ni;
    const R r = residual_u<FAST>(G, u, v, T, p, u_ant, fcon, flin, ii, jj);
    resu[G.at(ii, jj)] = r;
    acc += (double)r * (double)r;
  }
  const double s = block_sum(acc);
  const bool last = finish_norm(ns, s);
  if (last && outer.ctl && threadIdx.x == 0) ctl_outer_step(outer.ctl, outer.norms, outer.cond, outer.cond2);
}

// batched forms: work item i = (instance, block of kCellChunk cells)
template <bool FAST>
__global__ void __launch_bounds__(kCellChunk) correct_batch_kernel(const CellInst* __restrict__ inst,
                                                                   const int2* __restrict__ items, const int nitems,
                                                                   const int* __restrict__ active) {
  IXB_PDL_ENTRY();
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 wi = items[it];
    if (!active[wi.x]) continue;
    const CellInst& d = inst[wi.x];
    const int idx = wi.y * kCellChunk + threadIdx.x;
    if (idx < (d.G.mi - 1) * (d.G.nj - 1)) correct_cell<double, FAST>(d.G, d.u, d.v, d.p, d.pc, d.au, d.av, idx);
  }
}

template <bool FAST>
__global__ void __launch_bounds__(kCellChunk) residual_batch_kernel(const CellInst* __restrict__ inst,
                                                                    const int2* __restrict__ items, const int nitems,
                                                                    const int* __restrict__ active,
                                                                    const BatchNorm bn) {
  IXB_PDL_ENTRY();
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 wi = items[it];
    if (!active[wi.x]) continue;
    const CellInst& d = inst[wi.x];
    const int ni = d.G.mi - 2;
    const int idx = wi.y * kCellChunk + threadIdx.x;
    double acc = 0.0;
    if (idx < ni * (d.G.nj - 1)) {
      const int ii = 2 + idx % ni, jj = 2 + idx / ni;
      const double r = residual_u<FAST>(d.G, d.u, d.v, d.T, d.p, d.u_ant, d.fcon, d.flin, ii, jj);
      d.resu[d.G.at(ii, jj)] = r;
      acc = r * r;
    }
    finish_item_norm(bn, wi.x, d.first, d.count, it, block_sum(acc));
  }
}

cudaError_t correct_batch_launch(const CellInst* inst, const int2* items, int nitems, const int* active, int fast,
                                 cudaStream_t st) {
  const int grid = std::max(1, std::min(nitems, 148 * 16));
  if (fast) return launch_k(correct_batch_kernel<true>, grid, kCellChunk, 0, st, inst, items, nitems, active);
  return launch_k(correct_batch_kernel<false>, grid, kCellChunk, 0, st, inst, items, nitems, active);
}

cudaError_t residual_batch_launch(const CellInst* inst, const int2* items, int nitems, const int* active,
                                  const BatchNorm& bn, int fast, cudaStream_t st) {
  const int grid = std::max(1, std::min(nitems, 148 * 8));
  if (fast) return launch_k(residual_batch_kernel<true>, grid, kCellChunk, 0, st, inst, items, nitems, active, bn);
  return launch_k(residual_batch_kernel<false>, grid, kCellChunk, 0, st, inst, items, nitems, active, bn);
}

// ---------------------------------------------------------------------------
// Nusselt number on a wall (nusselt_promedio_y, source/mod_postproceso.f90:100-215,
// and its vertical-wall counterpart).  out2[0] = wall at index 1, out2[1] =
// wall at the last index.  With `quirk` set (the reference rule) the
// wall-normal derivative is known only on k0..k1 and reads as 0 beyond, as
// derivada does in the reference; the vertical-wall extension evaluates it
// on every node the panels touch.
//
// The panels' terms are evaluated in parallel (one panel per thread, in
// chunks of kNuThreads), then one thread per wall adds them in panel order
// with the reference's left-to-right accumulation, so the value equals the
// serial evaluation bit for bit.  With `mon` set (the Nusselt monitor of
// ixb_simple_converge, inside the loop graph) the wall and panel range come
// from the monitor's fields, and thread 0 applies the monitor's stopping
// test to the result, setting the monitor loop's condition `cond`.
// ---------------------------------------------------------------------------
constexpr int kNuThreads = 256;

__global__ void __launch_bounds__(kNuThreads)
    nusselt_kernel(const Geo<double> G, const double* __restrict__ T, const double* __restrict__ xp,
                   const double* __restrict__ yp, int vertical, int k0, int k1, double* __restrict__ out2, Ctl* mon,
                   cudaGraphConditionalHandle cond) {
  __shared__ double terms[2][3][kNuThreads];
  if (mon) {
    vertical = mon->mon_vertical;
    k0 = mon->mon_k0;
    k1 = mon->mon_k1;
  }
  const int quirk = vertical ? 0 : 1;
  const double* along = vertical ? yp : xp;  // 1-based
  const double* across = vertical ? xp : yp;
  const int n_across = vertical ? G.mi + 1 : G.nj + 1;
  auto f = [&](int k, int l) { return vertical ? T[G.at(l, k)] : T[G.at(k, l)]; };
  const int npan = (k1 - k0) / 2 + 1;
  const int tid = threadIdx.x;
  const int my_wall = tid == 0 ? 0 : 1;  // the summing threads: 0 (wall 0) and 32 (wall 1)
  double acc = 0.0;
  for (int base = 0; base < npan; base += kNuThreads) {
    const int pnl = base + tid;
    if (pnl < npan) {
      for (int wall = 0; wall < 2; ++wall) {
        double t[3];
        nusselt_panel(f, along, across, n_across, wall, quirk, k1, k0 + 2 * pnl, t);
        terms[wall][0][tid] = t[0];
        terms[wall][1][tid] = t[1];
        terms[wall][2][tid] = t[2];
      }
    }
    __syncthreads();
    if (tid == 0 || tid == 32) {
      const int cnt = min(kNuThreads, npan - base);
      for (int q = 0; q < cnt; ++q) acc = acc + terms[my_wall][0][q] + terms[my_wall][1][q] + terms[my_wall][2][q];
    }
    __syncthreads();
  }
  if (tid == 0 || tid == 32) out2[my_wall] = -acc;
  __syncthreads();
  if (mon && tid == 0) ctl_monitor_step(mon, out2, cond);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
int max_sweep_lines(int mi, int nj) { return std::max(mi, nj) + 2; }

SweepShape sweep_shape(int eq, int mi, int nj, int real_bytes, int tl, int g) {
  SweepShape s{};
  switch (eq) {
    case EQ_UY: s.n = nj + 1; s.line_lo = 2; s.line_hi = mi - 1; s.nfull = mi; break;
    case EQ_UX: s.n = mi; s.line_lo = 2; s.line_hi = nj; s.nfull = nj + 1; break;
    case EQ_VY: s.n = nj; s.line_lo = 2; s.line_hi = mi; s.nfull = mi + 1; break;
    case EQ_VX: s.n = mi + 1; s.line_lo = 2; s.line_hi = nj - 1; s.nfull = nj; break;
    case EQ_PY: s.n = nj + 1; s.line_lo = 2; s.line_hi = mi; s.nfull = mi + 1; break;
    case EQ_PX: s.n = mi + 1; s.line_lo = 2; s.line_hi = nj; s.nfull = nj + 1; break;
    case EQ_TY: s.n = nj + 1; s.line_lo = 2; s.line_hi = mi; s.nfull = mi + 1; break;
    default:    s.n = mi + 1; s.line_lo = 2; s.line_hi = nj; s.nfull = nj + 1; break;
  }
  s.tl = tl;
  s.g = g;
  s.nt = tl * g;
  s.m = std::max(3, (s.n + g - 1) / g);
  s.mp = s.m | 1;
  s.rs = RS_PCR;
  s.smem = line_smem_elems(g, s.mp) * real_bytes * tl;
  s.grid = (s.nfull + tl - 1) / tl;
  return s;
}

#define IXB_EQ_SWITCH(...)                                  \
  switch (eq) {                                               \
    case EQ_UY: { constexpr int E_ = EQ_UY; __VA_ARGS__; }           \
    case EQ_UX: { constexpr int E_ = EQ_UX; __VA_ARGS__; }           \
    case EQ_VY: { constexpr int E_ = EQ_VY; __VA_ARGS__; }           \
    case EQ_VX: { constexpr int E_ = EQ_VX; __VA_ARGS__; }           \
    case EQ_PY: { constexpr int E_ = EQ_PY; __VA_ARGS__; }           \
    case EQ_PX: { constexpr int E_ = EQ_PX; __VA_ARGS__; }           \
    case EQ_TY: { constexpr int E_ = EQ_TY; __VA_ARGS__; }           \
    default: { constexpr int E_ = EQ_TX; __VA_ARGS__; }              \
  }

// Orientation and defect-correction flag of the line solve of sweep `eq`.
static bool eq_is_x(int eq) { return (eq & 1) != 0; }
static bool eq_dc(int eq, int solver) { return solver == SOLVER_MIXED && eq != EQ_PY && eq != EQ_PX; }

int sweep_occupancy(int eq, int solver, const SweepShape& s) {
  return solve_blocks_per_sm(solver, eq_is_x(eq), eq_dc(eq, solver), s);
}

// Fused sweeps are on unless IXB_SPLIT=1 (the two-kernel form, for
// comparison).
bool fused_enabled() {
  static const bool on = [] {
    const char* e = getenv("IXB_SPLIT");
    return !(e && e[0] == '1');
  }();
  return on;
}

// Fused sweeps ask for a shared-memory carveout sized to one wave of their
// CTAs unless IXB_CARVEOUT=0.
bool carveout_enabled() {
  static const bool on = [] {
    const char* e = getenv("IXB_CARVEOUT");
    return !(e && e[0] == '0');
  }();
  return on;
}

bool pdl_enabled() {
  static const bool on = [] {
    const char* e = getenv("IXB_PDL");
    return e && e[0] == '1';
  }();
  return on;
}

// The shared-memory opt-in is a per-device function attribute, so it is set
// once per device (under a lock: handles may be created from several threads).
cudaError_t sweep_set_smem_limits() {
  constexpr int kMaxDev = 64;
  static bool done[kMaxDev] = {};
  static std::mutex mu;
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return cudaSuccess;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  e = solve_set_smem_limits(optin - 1024);  // room for the static reduction buffers
  if (e == cudaSuccess) done[dev] = true;
  return e;
}

// One sweep: the cell-parallel assembly stages the rows of every solved
// line in `buf`, then the line solve writes the field.
cudaError_t launch_sweep_f64(int eq, int solver, const SweepShape& s, const Geo<double>& G,
                             const SweepIO<double>& io, const StageBuf& buf, cudaStream_t st,
                             const CtlRef& ctl, const ResidIO* rio) {
  cudaError_t e;
  const bool fused = fused_enabled() && fused_shape(eq, s.tl, s.g);
  if (rio && (eq != EQ_TX || !fused || !io.nrm0.partials)) return cudaErrorInvalidValue;
  if (fused) {
    // assembly and solve in one kernel where the launch shape allows it
    SolveIO so{};
    so.in = io.in; so.out = io.out; so.prev = io.prev; so.nrm0 = io.nrm0; so.ctl = ctl;
    so.LD = G.LD; so.m = s.m; so.mp = s.mp;
    if (rio) so.res = *rio;
    auto fx = [&](auto solver_c) -> cudaError_t {
      constexpr int SV = decltype(solver_c)::value;
      IXB_EQ_SWITCH(return fused_launch<E_, SV>(s, G, io, so, st))
    };
    if (solver == IXB_SOLVER_EXACT) e = fx(std::integral_constant<int, IXB_SOLVER_EXACT>{});
    else if (solver == SOLVER_MIXED) e = fx(std::integral_constant<int, SOLVER_MIXED>{});
    else e = fx(std::integral_constant<int, IXB_SOLVER_HYBRID>{});
    if (e != cudaErrorNotSupported) return e;
  }
  if (solver == IXB_SOLVER_EXACT) {
    auto f = [&]() -> cudaError_t { IXB_EQ_SWITCH(return assemble_launch<E_, IXB_SOLVER_EXACT>(s, G, io, buf, st)) };
    e = f();
  } else if (solver == SOLVER_MIXED) {
    auto f = [&]() -> cudaError_t { IXB_EQ_SWITCH(return assemble_launch<E_, SOLVER_MIXED>(s, G, io, buf, st)) };
    e = f();
  } else {
    auto f = [&]() -> cudaError_t { IXB_EQ_SWITCH(return assemble_launch<E_, IXB_SOLVER_HYBRID>(s, G, io, buf, st)) };
    e = f();
  }
  if (e != cudaSuccess) return e;
  SolveIO so{};
  so.coef = buf.base; so.stride = buf.stride; so.P = buf.P;
  so.in = io.in; so.out = io.out; so.prev = io.prev; so.nrm0 = io.nrm0; so.ctl = ctl;
  so.LD = G.LD; so.m = s.m; so.mp = s.mp;
  return solve_launch(solver, eq_is_x(eq), eq_dc(eq, solver), s, so, st);
}

cudaError_t launch_preset_f64(double* pc, size_t n, const CtlRef& gate, cudaStream_t st) {
  const int grid = (int)std::min<size_t>((n + 255) / 256, 148 * 4);
  return launch_k(preset_kernel, grid, 256, 0, st, pc, n, gate);
}

cudaError_t launch_correct_f64(const Geo<double>& G, double* u, double* v, double* p, const double* pc,
                               const double* au, const double* av, int fast, cudaStream_t st, const CtlRef& gate) {
  const int total = (G.mi - 1) * (G.nj - 1);
  const int bs = 256;
  const int grid = (total + bs - 1) / bs;
  if (fast) return launch_k(correct_kernel<double, true>, grid, bs, 0, st, G, u, v, p, pc, au, av, gate);
  return launch_k(correct_kernel<double, false>, grid, bs, 0, st, G, u, v, p, pc, au, av, gate);
}

int residual_grid(int mi, int nj) {
  const int total = (mi - 2) * (nj - 1);
  return std::max(1, std::min((total + 255) / 256, 148 * 8));
}

cudaError_t launch_residual_f64(const Geo<double>& G, const double* u, const double* v, const double* T,
                                const double* p, const double* u_ant, const double* fcon, const double* flin,
                                double* resu, NormSlot ns, int fast, cudaStream_t st, const CtlRef& outer) {
  const int grid = residual_grid(G.mi, G.nj);
  if (fast)
    return launch_k(residual_kernel<double, true>, grid, 256, 0, st, G, u, v, T, p, u_ant, fcon, flin, resu, ns,
                    outer);
  return launch_k(residual_kernel<double, false>, grid, 256, 0, st, G, u, v, T, p, u_ant, fcon, flin, resu, ns,
                  outer);
}

cudaError_t launch_nusselt_f64(const Geo<double>& G, const double* T, const double* xp, const double* yp,
                               int vertical, int k0, int k1, double* out2, cudaStream_t st, Ctl* mon,
                               cudaGraphConditionalHandle cond) {
  nusselt_kernel<<<1, kNuThreads, 0, st>>>(G, T, xp, yp, vertical, k0, k1, out2, mon, cond);
  return cudaGetLastError();
}

}  // namespace ixb
