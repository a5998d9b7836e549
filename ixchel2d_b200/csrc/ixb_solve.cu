// ixb_solve.cu -- the line-solve half of a sweep: the rows staged by the
// assembly kernel (ixb_sweep.cuh) are read back coalesced, every line is
// solved in shared memory, and the solution is written to the field's
// ping-pong output buffer together with the pass norm ||new - prev||.
//
// Replaces the `tridiagonal` calls and the scatter of the solution into the
// field of each sweep (source/mod_solucionador.f90:25-47; e.g.
// source/main.f90:472-483).  A CTA owns TL adjacent lines with G threads per
// line (TL*G = 128 or 256): the partitioned Thomas + PCR solve of
// chunk_solve, or, for IXB_SOLVER_EXACT, the reference's sequential Thomas
// on one thread (bit-identical).  Lines outside the solved range are copied
// so that the output buffer holds the whole field.
#include <cuda_runtime.h>

#include <algorithm>

#include "ixb_ctl.cuh"
#include "ixb_internal.h"
#include "ixb_reduce.cuh"
#include "ixb_solve.cuh"

namespace ixb {
namespace {

// Lines L0 .. L0+TL-1 of one sweep: staged rows -> shared memory, then
// solve_lines (solve -> field).  Returns this thread's share of
// ||new - prev||^2.  Called by all threads of the CTA (it holds barriers).
template <class S, bool X, bool DC, bool EXACT, int TL, int G, int M>
__device__ __forceinline__ double solve_group(S* sm, const SolveIO& io, const int n, const int line_lo,
                                              const int line_hi, const int nfull, const int L0) {
  constexpr int NT = TL * G;
  const int m = M > 0 ? M : io.m;
  const int mp = M > 0 ? (M | 1) : io.mp;
  const int npad = G * m;
  const int LS = (int)line_smem_elems(G, mp);
  const int arr = G * mp;
  const S* ca = static_cast<const S*>(io.coef);
  const S* cb = ca + io.stride;
  const S* cc = cb + io.stride;
  const S* cd = cc + io.stride;

  // phase 1: staged rows -> chunk layout in shared memory (a warp reads 32
  // consecutive rows of one line); identity rows pad each line to G*m rows
#pragma unroll 4
  for (int it = 0; it < m; ++it) {
    const int idx = threadIdx.x + it * NT;
    const int l = TL == 1 ? 0 : idx / npad;
    const int r = idx - l * npad;
    const int L = L0 + l;
    S a = S(0), b = S(1), c = S(0), d = S(0);
    if (L >= line_lo && L <= line_hi && r < n) {
      const size_t o = (size_t)(L - line_lo) * io.P + r;
      a = ca[o]; b = cb[o]; c = cc[o]; d = cd[o];
    }
    const int ch = r / m;
    const int off = l * LS + ch * mp + (r - ch * m);
    sm[off] = a;
    sm[off + arr] = b;
    sm[off + 2 * arr] = c;
    sm[off + 3 * arr] = d;
  }
  __syncthreads();
  return solve_lines<S, X, DC, EXACT, TL, G, M>(sm, io, n, line_lo, line_hi, nfull, L0);
}

template <class S, bool X, bool DC, bool EXACT, int TL, int G, int M>
__global__ void __launch_bounds__(TL * G) solve_kernel(const SolveIO io, const int n, const int line_lo,
                                                       const int line_hi, const int nfull) {
  IXB_PDL_ENTRY();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const double acc = solve_group<S, X, DC, EXACT, TL, G, M>(reinterpret_cast<S*>(smem_raw), io, n, line_lo, line_hi,
                                                            nfull, 1 + blockIdx.x * TL);
  if (io.nrm0.partials) {
    const double s = block_sum(acc);
    const bool last = finish_norm(io.nrm0, s);
    if (last && io.ctl.ctl && threadIdx.x == 0) ctl_inner_step(io.ctl.ctl, io.ctl.norms, io.ctl.which, io.ctl.cond);
  }
}

// Batched line solve: work item i = (instance, line group) of items[i];
// a CTA walks the items grid-stride, skipping instances that no longer
// iterate; the pass norm is reduced per instance.
template <class S, bool X, bool DC, bool EXACT, int TL, int G>
__global__ void __launch_bounds__(TL * G) solve_batch_kernel(const SolveInst* __restrict__ inst,
                                                             const int2* __restrict__ items, const int nitems,
                                                             const int* __restrict__ active, const BatchNorm bn) {
  IXB_PDL_ENTRY();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 wi = items[it];
    if (!active[wi.x]) continue;  // uniform across the CTA
    const SolveInst& d = inst[wi.x];
    const double acc = solve_group<S, X, DC, EXACT, TL, G, 0>(reinterpret_cast<S*>(smem_raw), d.io, d.n, d.line_lo,
                                                              d.line_hi, d.nfull, 1 + wi.y * TL);
    if (bn.partials) finish_item_norm(bn, wi.x, d.first, d.count, it, block_sum(acc));
    __syncthreads();  // the next item reuses the shared memory
  }
}

// Launch shapes (lines per CTA x threads per line), kShapeList; 128 to 1024 threads.
#define IXB_SWEEP_SHAPES(X_) \
  X_(1, 128) X_(1, 256) X_(1, 512) X_(2, 64) X_(2, 128) X_(4, 32) X_(4, 64) X_(4, 128) X_(5, 64) X_(5, 128) \
  X_(6, 64) X_(6, 128) X_(8, 32) X_(8, 64) X_(8, 128) X_(16, 16) X_(16, 32)

template <class S, bool X, bool DC, bool EXACT>
struct SolveSet {
  static cudaError_t launch(const SweepShape& s, const SolveIO& io, cudaStream_t st) {
#define IXB_CASE_(TL_, G_)                                                                                    \
  if (s.tl == TL_ && s.g == G_) {                                                                             \
    if (!EXACT && s.m == 3)                                                                                   \
      return launch_k(solve_kernel<S, X, DC, EXACT, TL_, G_, 3>, s.grid, TL_ * G_, s.smem, st, io, s.n,       \
                      s.line_lo, s.line_hi, s.nfull);                                                         \
    return launch_k(solve_kernel<S, X, DC, EXACT, TL_, G_, 0>, s.grid, TL_ * G_, s.smem, st, io, s.n,         \
                    s.line_lo, s.line_hi, s.nfull);                                                           \
  }
    IXB_SWEEP_SHAPES(IXB_CASE_)
#undef IXB_CASE_
    return cudaErrorInvalidValue;
  }
  static int occupancy(const SweepShape& s) {
    int nb = 0;
    cudaError_t e = cudaErrorInvalidValue;
#define IXB_OCC_(TL_, G_)                                                                                     \
  if (s.tl == TL_ && s.g == G_) {                                                                             \
    if (!EXACT && s.m == 3)                                                                                   \
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, solve_kernel<S, X, DC, EXACT, TL_, G_, 3>,        \
                                                        TL_ * G_, s.smem);                                    \
    else                                                                                                      \
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, solve_kernel<S, X, DC, EXACT, TL_, G_, 0>,        \
                                                        TL_ * G_, s.smem);                                    \
  }
    IXB_SWEEP_SHAPES(IXB_OCC_)
#undef IXB_OCC_
    return e == cudaSuccess ? nb : 0;
  }
  static cudaError_t launch_batch(int tl, int g, size_t smem, const SolveInst* inst, const int2* items, int nitems,
                                  const int* active, const BatchNorm& bn, cudaStream_t st) {
#define IXB_BCASE_(TL_, G_)                                                                                \
  if (tl == TL_ && g == G_) {                                                                              \
    auto k = solve_batch_kernel<S, X, DC, EXACT, TL_, G_>;                                                 \
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);       \
    if (e != cudaSuccess) return e;                                                                        \
    int per_sm = 0, dev = 0, nsm = 0;                                                                      \
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, TL_ * G_, smem)) != cudaSuccess)    \
      return e;                                                                                            \
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;                                                \
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;  \
    if (per_sm < 1) return cudaErrorInvalidValue;                                                          \
    const int grid = std::max(1, std::min(nitems, per_sm * nsm));                                          \
    return launch_k(k, grid, TL_ * G_, smem, st, inst, items, nitems, active, bn);                         \
  }
    IXB_SWEEP_SHAPES(IXB_BCASE_)
#undef IXB_BCASE_
    return cudaErrorInvalidValue;
  }
  static cudaError_t limits(int bytes) {
    cudaError_t e = cudaSuccess;
    auto set = [&](auto k) {
      if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    };
#define IXB_SET_(TL_, G_)                                   \
  if (!EXACT) set(solve_kernel<S, X, DC, EXACT, TL_, G_, 3>); \
  set(solve_kernel<S, X, DC, EXACT, TL_, G_, 0>);
    IXB_SWEEP_SHAPES(IXB_SET_)
#undef IXB_SET_
    return e;
  }
};

// every (form, orientation, defect correction) combination the sweeps use
template <class F>
auto with_set(int form, bool x, bool dc, F&& f) {
  if (form == IXB_SOLVER_EXACT)
    return x ? f(SolveSet<double, true, false, true>{}) : f(SolveSet<double, false, false, true>{});
  if (form == SOLVER_MIXED) {
    if (dc) return x ? f(SolveSet<float, true, true, false>{}) : f(SolveSet<float, false, true, false>{});
    return x ? f(SolveSet<float, true, false, false>{}) : f(SolveSet<float, false, false, false>{});
  }
  return x ? f(SolveSet<double, true, false, false>{}) : f(SolveSet<double, false, false, false>{});
}

}  // namespace

cudaError_t solve_launch(int form, bool x, bool dc, const SweepShape& s, const SolveIO& io, cudaStream_t st) {
  return with_set(form, x, dc, [&](auto set) { return decltype(set)::launch(s, io, st); });
}

int solve_blocks_per_sm(int form, bool x, bool dc, const SweepShape& s) {
  return with_set(form, x, dc, [&](auto set) { return decltype(set)::occupancy(s); });
}

cudaError_t solve_batch_launch(int form, bool x, bool dc, int tl, int g, size_t smem, const SolveInst* inst,
                               const int2* items, int nitems, const int* active, const BatchNorm& bn,
                               cudaStream_t st) {
  return with_set(form, x, dc, [&](auto set) {
    return decltype(set)::launch_batch(tl, g, smem, inst, items, nitems, active, bn, st);
  });
}

cudaError_t solve_set_smem_limits(int bytes) {
  const int forms[3] = {IXB_SOLVER_HYBRID, IXB_SOLVER_EXACT, SOLVER_MIXED};
  for (int f : forms)
    for (int x = 0; x < 2; ++x)
      for (int dc = 0; dc < 2; ++dc) {
        if (dc && f != SOLVER_MIXED) continue;
        const cudaError_t e = with_set(f, x != 0, dc != 0, [&](auto set) { return decltype(set)::limits(bytes); });
        if (e != cudaSuccess) return e;
      }
  return cudaSuccess;
}

}  // namespace ixb
