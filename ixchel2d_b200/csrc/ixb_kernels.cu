// ixb_kernels.cu -- sm_100a kernels of the SIMPLE outer iteration.
//
// One fused kernel per line sweep replaces the reference's four OpenACC
// regions per sweep (assembly, impone_cond_frontera, tridiagonal, scatter;
// e.g. source/main.f90:420-484): a CTA owns TL adjacent lines, assembles
// their rows straight from the fields into shared memory (coalesced along
// ii), applies the boundary rows from a per-line table, solves each line
// with one warp, and writes the solution to the ping-pong output buffer,
// reducing the convergence norm of the pass on the way out.
#include <cuda_runtime.h>

#include <algorithm>

#include "ixb_internal.h"

namespace ixb {

// ---------------------------------------------------------------------------
// reductions (fixed order: deterministic run to run)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ double block_sum(double v) {
  __shared__ double red[32];
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (w == 0) {
    s = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
    s = warp_sum(s);
  }
  return s;  // valid in thread 0
}

// Publish this CTA's partial; the last CTA to arrive sums all partials in
// CTA order and stores sqrt(sum).
__device__ void finish_norm(const NormSlot& ns, double block_total) {
  __shared__ int is_last;
  if (threadIdx.x == 0) {
    ns.partials[blockIdx.x] = block_total;
    __threadfence();
    const unsigned prev = atomicAdd(ns.counter, 1u);
    is_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (is_last && threadIdx.x < 32) {
    __threadfence();
    double s = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) s += __ldcg(ns.partials + i);
    s = warp_sum(s);
    if (threadIdx.x == 0) {
      *ns.result = sqrt(s);
      *ns.counter = 0u;
    }
  }
}

// ---------------------------------------------------------------------------
// per-equation assembly dispatch
// ---------------------------------------------------------------------------
template <int EQ>
struct EqIsX { static constexpr bool value = (EQ & 1) != 0; };

template <class R, int EQ>
__device__ __forceinline__ Row<R> assemble_cell(const Geo<R>& G, const SweepIO<R>& io, int ii, int jj,
                                                double& acc_bo) {
  if constexpr (EQ == EQ_UY) {
    return assemble_uy(G, io, ii, jj);
  } else if constexpr (EQ == EQ_UX) {
    R au;
    Row<R> r = assemble_ux(G, io, ii, jj, au);
    io.aux[G.at(ii, jj)] = au;
    return r;
  } else if constexpr (EQ == EQ_VY) {
    return assemble_vy(G, io, ii, jj);
  } else if constexpr (EQ == EQ_VX) {
    R av;
    Row<R> r = assemble_vx(G, io, ii, jj, av);
    io.aux[G.at(ii, jj)] = av;
    return r;
  } else if constexpr (EQ == EQ_PY) {
    return assemble_py(G, io, ii, jj);
  } else if constexpr (EQ == EQ_PX) {
    R bo;
    Row<R> r = assemble_px(G, io, ii, jj, bo);
    io.aux[G.at(ii, jj)] = bo;
    acc_bo += (double)bo * (double)bo;
    return r;
  } else if constexpr (EQ == EQ_TY) {
    return assemble_ty(G, io, ii, jj);
  } else {
    return assemble_tx(G, io, ii, jj);
  }
}

// Boundary rows of impone_cond_frontera (source/mod_cond_frontera.f90:280-416):
// first row of a line: diri (0,1,0|val), neum (0,-1,1|val);
// last row: diri (0,1,0|val), neum (-1,1,0|val).  p' rows are hard-coded
// Dirichlet 0 (main.f90:789-800, 845-856).
template <class R>
__device__ __forceinline__ Row<R> bc_first_row(const BCEntry* t, int L) {
  if (!t) return Row<R>{R(0), R(1), R(0), R(0)};
  const BCEntry e = t[L];
  if (e.type == 2) return Row<R>{R(0), R(-1), R(1), R(e.val)};
  return Row<R>{R(0), R(1), R(0), R(e.val)};
}
template <class R>
__device__ __forceinline__ Row<R> bc_last_row(const BCEntry* t, int L) {
  if (!t) return Row<R>{R(0), R(1), R(0), R(0)};
  const BCEntry e = t[L];
  if (e.type == 2) return Row<R>{R(-1), R(1), R(0), R(e.val)};
  return Row<R>{R(0), R(1), R(0), R(e.val)};
}

// ---------------------------------------------------------------------------
// fused sweep kernel
// ---------------------------------------------------------------------------
template <class R, int EQ, int SOLVER, int TL>
__global__ void __launch_bounds__(512) sweep_kernel(const Geo<R> G, const SweepIO<R> io, const int n,
                                                    const int line_lo, const int line_hi, const int nfull) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sm = reinterpret_cast<R*>(smem_raw);
  constexpr bool X = EqIsX<EQ>::value;
  const int m = io.m, mp = io.mp;
  const int npad = 32 * m;
  const int chunk = 32 * mp;
  const int L0 = 1 + blockIdx.x * TL;
  const int NT = blockDim.x;
  double acc_bo = 0.0;

  // phase 1: assemble every row of the solved lines into shared memory
  for (int idx = threadIdx.x; idx < TL * npad; idx += NT) {
    int l, r;
    if (X) { l = idx / npad; r = idx - l * npad; }
    else { l = idx % TL; r = idx / TL; }
    const int L = L0 + l;
    if (L < line_lo || L > line_hi) continue;
    Row<R> row;
    if (r >= n) row = Row<R>{R(0), R(1), R(0), R(0)};  // identity padding
    else if (r == 0) row = bc_first_row<R>(io.bc_first, L);
    else if (r == n - 1) row = bc_last_row<R>(io.bc_last, L);
    else {
      const int ii = X ? r + 1 : L;
      const int jj = X ? L : r + 1;
      row = assemble_cell<R, EQ>(G, io, ii, jj, acc_bo);
    }
    const int lane = r / m;
    const int o = lane * mp + (r - lane * m);
    R* base = sm + l * 4 * chunk;
    base[o] = row.a;
    base[chunk + o] = row.b;
    base[2 * chunk + o] = row.c;
    base[3 * chunk + o] = row.d;
  }
  __syncthreads();

  // phase 2: one warp per line
  {
    const int w = threadIdx.x >> 5;
    if (w < TL) {
      const int L = L0 + w;
      if (L >= line_lo && L <= line_hi) {
        R* base = sm + w * 4 * chunk;
        if (SOLVER == IXB_SOLVER_EXACT) {
          if ((threadIdx.x & 31) == 0) thomas_exact(base, base + chunk, base + 2 * chunk, base + 3 * chunk, n, m, mp);
        } else {
          thomas_pcr_warp(base, base + chunk, base + 2 * chunk, base + 3 * chunk, m, mp);
        }
      }
    }
  }
  __syncthreads();

  // phase 3: write the new field (unsolved lines keep their values) and
  // accumulate ||new - prev|| over the interior rows of the solved lines
  double acc = 0.0;
  for (int idx = threadIdx.x; idx < TL * n; idx += NT) {
    int l, r;
    if (X) { l = idx / n; r = idx - l * n; }
    else { l = idx % TL; r = idx / TL; }
    const int L = L0 + l;
    if (L > nfull) continue;
    const int ii = X ? r + 1 : L;
    const int jj = X ? L : r + 1;
    const size_t g = G.at(ii, jj);
    R x;
    if (L >= line_lo && L <= line_hi) {
      const int lane = r / m;
      x = sm[l * 4 * chunk + 3 * chunk + lane * mp + (r - lane * m)];
      if (io.nrm0.partials && r >= 1 && r <= n - 2) {
        const double dv = (double)x - (io.prev ? (double)io.prev[g] : 0.0);
        acc += dv * dv;
      }
    } else {
      x = io.in ? io.in[g] : R(0);
    }
    io.out[g] = x;
  }
  if (io.nrm0.partials) {
    const double s = block_sum(acc);
    finish_norm(io.nrm0, s);
  }
  if (io.nrm1.partials) {
    const double s = block_sum(acc_bo);
    finish_norm(io.nrm1, s);
  }
}

// ---------------------------------------------------------------------------
// pressure and velocity correction, main.f90:931-962
// ---------------------------------------------------------------------------
template <class R>
__global__ void correct_kernel(const Geo<R> G, R* __restrict__ u, R* __restrict__ v, R* __restrict__ p,
                               const R* __restrict__ pc, const R* __restrict__ au, const R* __restrict__ av) {
  const int ni = G.mi - 1;  // ii = 2..mi
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int total = ni * (G.nj - 1);
  if (idx >= total) return;
  const int ii = 2 + idx % ni;
  const int jj = 2 + idx / ni;
  const size_t c0 = G.at(ii, jj);
  p[c0] = p[c0] + G.p_update * pc[c0];
  if (ii <= G.mi - 1) u[c0] = u[c0] + G.met(M_DYU, jj) * (pc[c0] - pc[G.at(ii + 1, jj)]) / au[c0];
  if (jj <= G.nj - 1) v[c0] = v[c0] + G.met(M_DXV, ii) * (pc[c0] - pc[G.at(ii, jj + 1)]) / av[c0];
}

// ---------------------------------------------------------------------------
// u residual and its norm, main.f90:1169-1199
// ---------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) residual_kernel(const Geo<R> G, const R* __restrict__ u,
                                                       const R* __restrict__ v, const R* __restrict__ T,
                                                       const R* __restrict__ p, const R* __restrict__ u_ant,
                                                       const R* __restrict__ fcon, const R* __restrict__ flin,
                                                       R* __restrict__ resu, NormSlot ns) {
  const int ni = G.mi - 2;  // ii = 2..mi-1
  const int total = ni * (G.nj - 1);
  double acc = 0.0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int ii = 2 + idx % ni;
    const int jj = 2 + idx / ni;
    const R r = residual_u(G, u, v, T, p, u_ant, fcon, flin, ii, jj);
    resu[G.at(ii, jj)] = r;
    acc += (double)r * (double)r;
  }
  const double s = block_sum(acc);
  finish_norm(ns, s);
}

// ---------------------------------------------------------------------------
// Nusselt number on a wall (nusselt_promedio_y, source/mod_postproceso.f90:100-215,
// and its vertical-wall counterpart); one thread, serial like the reference.
// out2[0] = wall at index 1, out2[1] = wall at the last index.  With
// `quirk` set (the reference rule) the wall-normal derivative is known only
// on k0..k1 and reads as 0 beyond, as derivada does in the reference; the
// vertical-wall extension evaluates it on every node the panels touch.
// ---------------------------------------------------------------------------
__global__ void nusselt_kernel(const Geo<double> G, const double* __restrict__ T, const double* __restrict__ xp,
                               const double* __restrict__ yp, int vertical, int quirk, int k0, int k1,
                               double* __restrict__ out2) {
  if (threadIdx.x != 0) return;
  const double* along = vertical ? yp : xp;   // 1-based
  const double* across = vertical ? xp : yp;
  const int n_across = vertical ? G.mi + 1 : G.nj + 1;
  auto f = [&](int k, int l) { return vertical ? T[G.at(l, k)] : T[G.at(k, l)]; };
  for (int wall = 0; wall < 2; ++wall) {
    const int jj = wall == 0 ? 1 : n_across - 2;
    double nu = 0.0;
    for (int ii = k0; ii <= k1; ii += 2) {
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
      nu = nu + alpha / 3.0 * (x_2 * x_2 * x_2 - x_o * x_o * x_o) + beta / 2.0 * (x_2 * x_2 - x_o * x_o) +
           gamma * (x_2 - x_o);
    }
    out2[wall] = -nu;
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
int max_sweep_lines(int mi, int nj) { return std::max(mi, nj) + 2; }

SweepShape sweep_shape(int eq, int mi, int nj, int real_bytes, int tl_override, int nt_override) {
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
  s.m = std::max(3, (s.n + 31) / 32);
  s.mp = s.m | 1;
  const bool x = (eq & 1) != 0;
  int tl = x ? 1 : 4;
  if (tl_override > 0) tl = tl_override;
  const size_t per_line = (size_t)4 * 32 * s.mp * real_bytes;
  while (tl > 1 && per_line * tl > 200 * 1024) tl >>= 1;
  s.tl = tl;
  int nt = x ? (s.n > 256 ? 256 : 128) : std::max(128, 32 * tl);
  if (nt_override > 0) nt = nt_override;
  nt = std::max(nt, 32 * tl);
  nt = std::min(nt, 512);
  s.nt = nt;
  s.smem = per_line * tl;
  s.grid = (s.nfull + tl - 1) / tl;
  return s;
}

template <class R, int EQ, int SOLVER, int TL>
static cudaError_t launch_one(const SweepShape& s, const Geo<R>& G, const SweepIO<R>& io, cudaStream_t st) {
  sweep_kernel<R, EQ, SOLVER, TL><<<s.grid, s.nt, s.smem, st>>>(G, io, s.n, s.line_lo, s.line_hi, s.nfull);
  return cudaGetLastError();
}

// Raise the dynamic shared-memory limit of every sweep instantiation once
// (outside any stream capture).
template <class R, int EQ, int SOLVER>
static cudaError_t smem_limit_eq(int bytes) {
  cudaError_t e = cudaSuccess;
  auto set = [&](auto k) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  };
  set(sweep_kernel<R, EQ, SOLVER, 1>);
  set(sweep_kernel<R, EQ, SOLVER, 2>);
  set(sweep_kernel<R, EQ, SOLVER, 4>);
  set(sweep_kernel<R, EQ, SOLVER, 8>);
  return e;
}
template <class R, int SOLVER>
static cudaError_t smem_limit_all(int bytes) {
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = smem_limit_eq<R, EQ_UY, SOLVER>(bytes);
  if (e == cudaSuccess) e = smem_limit_eq<R, EQ_UX, SOLVER>(bytes);
  if (e == cudaSuccess) e = smem_limit_eq<R, EQ_VY, SOLVER>(bytes);
  if (e == cudaSuccess) e = smem_limit_eq<R, EQ_VX, SOLVER>(bytes);
  if (e == cudaSuccess) e = smem_limit_eq<R, EQ_PY, SOLVER>(bytes);
  if (e == cudaSuccess) e = smem_limit_eq<R, EQ_PX, SOLVER>(bytes);
  if (e == cudaSuccess) e = smem_limit_eq<R, EQ_TY, SOLVER>(bytes);
  if (e == cudaSuccess) e = smem_limit_eq<R, EQ_TX, SOLVER>(bytes);
  return e;
}
cudaError_t sweep_set_smem_limits() {
  static int done = 0;
  if (done) return cudaSuccess;
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  const int bytes = optin - 1024;  // leave room for the static reduction buffers
  e = smem_limit_all<double, IXB_SOLVER_HYBRID>(bytes);
  if (e == cudaSuccess) e = smem_limit_all<double, IXB_SOLVER_EXACT>(bytes);
  if (e == cudaSuccess) done = 1;
  return e;
}

template <class R, int EQ, int SOLVER>
static cudaError_t launch_tl(const SweepShape& s, const Geo<R>& G, const SweepIO<R>& io, cudaStream_t st) {
  switch (s.tl) {
    case 1: return launch_one<R, EQ, SOLVER, 1>(s, G, io, st);
    case 2: return launch_one<R, EQ, SOLVER, 2>(s, G, io, st);
    case 4: return launch_one<R, EQ, SOLVER, 4>(s, G, io, st);
    case 8: return launch_one<R, EQ, SOLVER, 8>(s, G, io, st);
    default: return cudaErrorInvalidValue;
  }
}

template <class R, int SOLVER>
static cudaError_t launch_eq(int eq, const SweepShape& s, const Geo<R>& G, const SweepIO<R>& io, cudaStream_t st) {
  switch (eq) {
    case EQ_UY: return launch_tl<R, EQ_UY, SOLVER>(s, G, io, st);
    case EQ_UX: return launch_tl<R, EQ_UX, SOLVER>(s, G, io, st);
    case EQ_VY: return launch_tl<R, EQ_VY, SOLVER>(s, G, io, st);
    case EQ_VX: return launch_tl<R, EQ_VX, SOLVER>(s, G, io, st);
    case EQ_PY: return launch_tl<R, EQ_PY, SOLVER>(s, G, io, st);
    case EQ_PX: return launch_tl<R, EQ_PX, SOLVER>(s, G, io, st);
    case EQ_TY: return launch_tl<R, EQ_TY, SOLVER>(s, G, io, st);
    case EQ_TX: return launch_tl<R, EQ_TX, SOLVER>(s, G, io, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_sweep_f64(int eq, int solver, const SweepShape& s, const Geo<double>& G,
                             const SweepIO<double>& io, cudaStream_t st) {
  if (solver == IXB_SOLVER_EXACT) return launch_eq<double, IXB_SOLVER_EXACT>(eq, s, G, io, st);
  return launch_eq<double, IXB_SOLVER_HYBRID>(eq, s, G, io, st);
}

cudaError_t launch_correct_f64(const Geo<double>& G, double* u, double* v, double* p, const double* pc,
                               const double* au, const double* av, cudaStream_t st) {
  const int total = (G.mi - 1) * (G.nj - 1);
  const int bs = 256;
  correct_kernel<double><<<(total + bs - 1) / bs, bs, 0, st>>>(G, u, v, p, pc, au, av);
  return cudaGetLastError();
}

int residual_grid(int mi, int nj) {
  const int total = (mi - 2) * (nj - 1);
  return std::max(1, std::min((total + 255) / 256, 148 * 8));
}

cudaError_t launch_residual_f64(const Geo<double>& G, const double* u, const double* v, const double* T,
                                const double* p, const double* u_ant, const double* fcon, const double* flin,
                                double* resu, NormSlot ns, cudaStream_t st) {
  residual_kernel<double><<<residual_grid(G.mi, G.nj), 256, 0, st>>>(G, u, v, T, p, u_ant, fcon, flin, resu, ns);
  return cudaGetLastError();
}

cudaError_t launch_nusselt_f64(const Geo<double>& G, const double* T, const double* xp, const double* yp,
                               int vertical, int k0, int k1, double* out2, cudaStream_t st) {
  nusselt_kernel<<<1, 32, 0, st>>>(G, T, xp, yp, vertical, vertical ? 0 : 1, k0, k1, out2);
  return cudaGetLastError();
}

}  // namespace ixb
