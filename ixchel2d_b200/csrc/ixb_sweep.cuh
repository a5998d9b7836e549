// ixb_sweep.cuh -- the assembly half of a line sweep: every row of the
// sweep's tridiagonal systems (coefficients, boundary rows, and for the
// mixed-precision form the binary64 defect-correction residual) evaluated
// cell-parallel and staged line-major for the line solver (ixb_solve.cu).
// Included by the per-equation translation units ixb_sweep_<eq>[_fast|_mixed].cu.
//
// A sweep of the reference is four OpenACC regions (assembly,
// impone_cond_frontera, tridiagonal, scatter; e.g. source/main.f90:420-484).
// Here it is two kernels: this cell-parallel assembly (one thread per cell,
// loads coalesced along ii, enough warps to hide the latency of its ~30
// stencil loads) writing rows a,b,c,d of every solved line contiguously, and
// the partitioned line solve that reads them back coalesced.  y-sweep tiles
// are transposed through shared memory so that both the field reads and the
// row writes are coalesced.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "ixb_ctl.cuh"
#include "ixb_internal.h"
#include "ixb_reduce.cuh"
#include "ixb_solve.cuh"

namespace ixb {

// ---------------------------------------------------------------------------
// per-equation assembly dispatch
// ---------------------------------------------------------------------------

// Row of cell (ii,jj); the side outputs (au, av, b_o and the b_o norm) are
// written only when `keep` is set.
template <class R, int EQ, bool FAST, class F>
__device__ __forceinline__ Row<R> assemble_cell(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj,
                                                double& acc_bo, bool keep) {
  if constexpr (EQ == EQ_UY) {
    return assemble_uy<FAST>(G, io, ii, jj);
  } else if constexpr (EQ == EQ_UX) {
    R au;
    Row<R> r = assemble_ux<FAST>(G, io, ii, jj, au);
    if (keep) io.aux[G.at(ii, jj)] = F(au);
    return r;
  } else if constexpr (EQ == EQ_VY) {
    return assemble_vy<FAST>(G, io, ii, jj);
  } else if constexpr (EQ == EQ_VX) {
    R av;
    Row<R> r = assemble_vx<FAST>(G, io, ii, jj, av);
    if (keep) io.aux[G.at(ii, jj)] = F(av);
    return r;
  } else if constexpr (EQ == EQ_PY) {
    return assemble_py<FAST>(G, io, ii, jj);
  } else if constexpr (EQ == EQ_PX) {
    F bo;
    Row<R> r = assemble_px<FAST>(G, io, ii, jj, bo);
    if (keep) {
      io.aux[G.at(ii, jj)] = bo;
      acc_bo += (double)bo * (double)bo;
    }
    return r;
  } else if constexpr (EQ == EQ_TY) {
    return assemble_ty<FAST>(G, io, ii, jj);
  } else {
    return assemble_tx<FAST>(G, io, ii, jj);
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
// assembly kernel
// ---------------------------------------------------------------------------
// Row of line L, position r (0-based along the line) of sweep EQ, or an
// identity row outside the line.  Rows outside the interior are assembled
// at the nearest interior cell and then replaced, so every load is in bounds
// and no branch separates a thread's loads.
template <int EQ, int SOLVER>
__device__ __forceinline__ Row<double> staged_row(
    const Geo<double>& Gm, const SweepIO<double>& io, int L, int r, int n, int line_lo,
    int line_hi, bool valid, double& acc_bo) {
  using ST = SweepTypes<SOLVER, EQ>;
  using A = double;
  constexpr bool X = EqIsX<EQ>::value;
  const int Lc = min(max(L, line_lo), line_hi);
  const int rc = min(max(r, 1), n - 2);
  const bool interior = valid && r >= 1 && r <= n - 2;
  Row<A> row = assemble_cell<A, EQ, SOLVER != IXB_SOLVER_EXACT>(Gm, io, X ? rc + 1 : Lc, X ? Lc : rc + 1, acc_bo,
                                                                interior);
  const Row<A> first = bc_first_row<A>(io.bc_first, Lc);
  const Row<A> last = bc_last_row<A>(io.bc_last, Lc);
  if (r == 0) row = first;
  else if (r == n - 1) row = last;
  if constexpr (ST::DC) {
    // defect correction: the row's binary64 residual at the current values
    const int rr = min(max(r, 0), n - 1);
    const int g = Gm.at(X ? rr + 1 : Lc, X ? Lc : rr + 1);
    const int step = X ? 1 : Gm.LD;
    const double xm = __ldg(io.in + (rr > 0 ? g - step : g));
    const double x0 = __ldg(io.in + g);
    const double xp = __ldg(io.in + (rr < n - 1 ? g + step : g));
    double res = fma(-row.b, x0, row.d);
    res = fma(-row.a, xm, res);
    res = fma(-row.c, xp, res);
    row.d = res;
  }
  if constexpr (ST::MIX) {
    // unit diagonal before the binary32 staging; the solution is unchanged
    // (a Newton-refined reciprocal: the scaled row is rounded to binary32)
    const double sc = fast_rcp(row.b);
    row.a *= sc;
    row.c *= sc;
    row.d *= sc;
    row.b = 1.0;
  }
  return row;
}

// One tile of the assembly of sweep EQ: rows of lines line_lo..line_hi
// written to `co` (line L at (L - line_lo) * P).  Called by all threads of
// the CTA (a y tile holds barriers around its shared-memory transpose).
template <int EQ, int SOLVER>
__device__ __forceinline__ void assemble_tile(const Geo<double>& G_,
                                              const SweepIO<double>& io,
                                              const Coef<typename SweepTypes<SOLVER, EQ>::S>& co, const int n,
                                              const int line_lo, const int line_hi, const int tile, double& acc_bo,
                                              typename SweepTypes<SOLVER, EQ>::S (*tile_s)[kAsmYR][kAsmYL + 1]) {
  using S = typename SweepTypes<SOLVER, EQ>::S;
  constexpr bool X = EqIsX<EQ>::value;
  if constexpr (X) {
    const int tr_n = (n + kAsmXR - 1) / kAsmXR;
    const int tl = tile / tr_n, tr = tile - tl * tr_n;
    const int r = tr * kAsmXR + (threadIdx.x % kAsmXR);
#pragma unroll
    for (int u = 0; u < kAsmCPT; ++u) {
      const int L = line_lo + tl * kAsmXL + threadIdx.x / kAsmXR + u * (kAsmThreads / kAsmXR);
      const bool valid = r < n && L <= line_hi;
      const auto row = staged_row<EQ, SOLVER>(G_, io, L, r, n, line_lo, line_hi, valid, acc_bo);
      if (valid) {
        const size_t o = (size_t)(L - line_lo) * co.P + r;
        co.a[o] = S(row.a); co.b[o] = S(row.b); co.c[o] = S(row.c); co.d[o] = S(row.d);
      }
    }
  } else {
    const int nl = line_hi - line_lo + 1;
    const int tl_n = (nl + kAsmYL - 1) / kAsmYL;
    const int tr = tile / tl_n, tl = tile - tr * tl_n;
    const int lo = threadIdx.x % kAsmYL;
    const int L = line_lo + tl * kAsmYL + lo;  // adjacent ii in a warp: coalesced field reads
#pragma unroll
    for (int u = 0; u < kAsmCPT; ++u) {
      const int ro = threadIdx.x / kAsmYL + u * (kAsmThreads / kAsmYL);
      const int r = tr * kAsmYR + ro;
      const bool valid = r < n && L <= line_hi;
      const auto row = staged_row<EQ, SOLVER>(G_, io, L, r, n, line_lo, line_hi, valid, acc_bo);
      tile_s[0][ro][lo] = S(row.a); tile_s[1][ro][lo] = S(row.b);
      tile_s[2][ro][lo] = S(row.c); tile_s[3][ro][lo] = S(row.d);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kAsmCPT; ++u) {  // kAsmYR-row runs of one line
      const int q = threadIdx.x + u * kAsmThreads;
      const int wl = q / kAsmYR, wr = q % kAsmYR;
      const int Lw = line_lo + tl * kAsmYL + wl, rw = tr * kAsmYR + wr;
      if (Lw <= line_hi && rw < n) {
        const size_t o = (size_t)(Lw - line_lo) * co.P + rw;
        co.a[o] = tile_s[0][wr][wl]; co.b[o] = tile_s[1][wr][wl];
        co.c[o] = tile_s[2][wr][wl]; co.d[o] = tile_s[3][wr][wl];
      }
    }
    __syncthreads();
  }
}

// Assemble the rows of lines line_lo..line_hi of sweep EQ into `co`.
// Grid-stride over tiles; the b_o norm (p'-x) is reduced over the grid.
template <int EQ, int SOLVER>
__global__ void __launch_bounds__(kAsmThreads)
    assemble_kernel(const Geo<double> G_, const SweepIO<double> io,
                    const Coef<typename SweepTypes<SOLVER, EQ>::S> co, const int n, const int line_lo,
                    const int line_hi) {
  IXB_PDL_ENTRY();
  using S = typename SweepTypes<SOLVER, EQ>::S;
  __shared__ S tile_s[4][kAsmYR][kAsmYL + 1];
  const int ntiles = asm_tiles(EqIsX<EQ>::value, n, line_hi - line_lo + 1);
  double acc_bo = 0.0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    assemble_tile<EQ, SOLVER>(G_, io, co, n, line_lo, line_hi, tile, acc_bo, tile_s);
  if (io.nrm1.partials) {
    const double s = block_sum(acc_bo);
    finish_norm(io.nrm1, s);
  }
}

// Batched assembly: work item i = (instance, tile) of items[i]; a CTA walks
// the items grid-stride, skipping instances that no longer iterate.  The
// b_o norm is reduced per instance over its items (finish_item_norm).
template <int EQ, int SOLVER>
__global__ void __launch_bounds__(kAsmThreads)
    assemble_batch_kernel(const AsmInst<typename SweepTypes<SOLVER, EQ>::S>*
                              __restrict__ inst,
                          const int2* __restrict__ items, const int nitems, const int* __restrict__ active,
                          const BatchNorm bn) {
  IXB_PDL_ENTRY();
  using S = typename SweepTypes<SOLVER, EQ>::S;
  __shared__ S tile_s[4][kAsmYR][kAsmYL + 1];
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 wi = items[it];
    if (!active[wi.x]) continue;  // uniform across the CTA
    const auto& d = inst[wi.x];
    double acc_bo = 0.0;
    assemble_tile<EQ, SOLVER>(d.G, d.io, d.co, d.n, d.line_lo, d.line_hi, wi.y, acc_bo, tile_s);
    if (bn.partials) finish_item_norm(bn, wi.x, d.first, d.count, it, block_sum(acc_bo));
  }
}

template <int EQ, int SOLVER>
cudaError_t assemble_batch_launch(const void* inst, const int2* items, int nitems, const int* active,
                                  const BatchNorm& bn, cudaStream_t st) {
  using ST = SweepTypes<SOLVER, EQ>;
  const int grid = std::max(1, std::min(nitems, kAsmGridCap * 4));
  return launch_k(assemble_batch_kernel<EQ, SOLVER>, grid, kAsmThreads, 0, st,
                  static_cast<const AsmInst<typename ST::S>*>(inst), items, nitems, active, bn);
}

template <int EQ, int SOLVER>
cudaError_t assemble_launch(const SweepShape& s, const Geo<double>& G, const SweepIO<double>& io,
                            const StageBuf& buf, cudaStream_t st) {
  using S = typename SweepTypes<SOLVER, EQ>::S;
  Coef<S> co;
  S* base = static_cast<S*>(buf.base);
  co.a = base; co.b = base + buf.stride; co.c = base + 2 * buf.stride; co.d = base + 3 * buf.stride;
  co.P = buf.P;
  const int tiles = asm_tiles(EqIsX<EQ>::value, s.n, s.line_hi - s.line_lo + 1);
  const int grid = std::max(1, std::min(tiles, kAsmGridCap));
  return launch_k(assemble_kernel<EQ, SOLVER>, grid, kAsmThreads, 0, st, G, io, co, s.n, s.line_lo, s.line_hi);
}

// ---------------------------------------------------------------------------
// Fused sweep: a CTA assembles the rows of its TL lines straight into the
// chunk layout of the line solve in shared memory, solves and writes the
// lines, then finishes the b_o norm (p'-x) and the pass norm with its loop
// test.  One launch per sweep instead of two, and no staging of the rows
// through global memory.  x-lines: consecutive threads take consecutive
// cells of a line; y-lines: consecutive threads take the TL adjacent lines
// of a row, so the field reads stay coalesced.
// ---------------------------------------------------------------------------
// Rows of lines L0 .. L0+TL-1 of sweep EQ assembled into the chunk layout of
// solve_lines (m rows per chunk at pitch mp); identity rows pad each line to
// G*m rows.  Returns nothing; acc_bo collects the b_o norm (p'-x).
template <int EQ, int SOLVER, int TL, int G, int M>
__device__ __forceinline__ void fused_assemble(typename SweepTypes<SOLVER, EQ>::S* sm, const Geo<double>& G_,
                                               const SweepIO<double>& io, const int m, const int mp, const int n,
                                               const int line_lo, const int line_hi, const int L0,
                                               double& acc_bo) {
  using S = typename SweepTypes<SOLVER, EQ>::S;
  constexpr bool X = EqIsX<EQ>::value;
  constexpr int NT = TL * G;
  const int npad = G * m;
  const int LS = (int)line_smem_elems(G, mp);
  const int arr = G * mp;
#pragma unroll
  for (int it = 0; it < (M > 0 ? M : m); ++it) {  // with M > 0 a thread's M cells are assembled together
    const int idx = threadIdx.x + it * NT;
    int l, r;
    if (X) { l = TL == 1 ? 0 : idx / npad; r = idx - l * npad; }
    else if (M > 0) {
      // y-lines with a compile-time chunk: each thread assembles the M
      // consecutive rows of its own chunk, so neighbouring rows' stencil
      // loads (row jj+1 of one cell is row jj of the next) repeat within
      // the thread and the compiler may keep them in registers
      l = threadIdx.x % TL;
      r = (threadIdx.x / TL) * M + it;
    } else { l = idx % TL; r = idx / TL; }
    const int L = L0 + l;
    const bool valid = L >= line_lo && L <= line_hi && r < n;
    // padding rows and unsolved lines: identity rows, nothing to assemble
    // (assembling them too, branch-free, and replacing them measured slower)
    const Row<double> row = valid ? staged_row<EQ, SOLVER>(G_, io, L, r, n, line_lo, line_hi, true, acc_bo)
                                  : Row<double>{0.0, 1.0, 0.0, 0.0};
    const int ch = r / m;
    const int off = l * LS + ch * mp + (r - ch * m);
    sm[off] = S(row.a);
    sm[off + arr] = S(row.b);
    sm[off + 2 * arr] = S(row.c);
    sm[off + 3 * arr] = S(row.d);
  }
}

// u residual (residuo_u) of row jj = L0 of a fused T-x sweep (one line per
// CTA): cells ii = 2..mi-1, m per thread (G*m >= mi+1 rows of the line);
// with a compile-time m the cells' loads are independent and issued
// together.  T: the temperature the residual's buoyancy term reads (written
// earlier in this kernel when T_WRITTEN).  Returns this thread's sum of
// squares.
template <bool FAST, bool T_WRITTEN, int G, int M>
__device__ __forceinline__ double tx_residual_row(const Geo<double>& G_, const ResidIO& r, const double* T, int m,
                                                  int L0) {
  double acc = 0.0;
  if (L0 < 2 || L0 > G_.nj) return acc;
#pragma unroll (M > 0 ? M : 3)
  for (int k = 0; k < (M > 0 ? M : m); ++k) {
    const int ii = 2 + (int)threadIdx.x + k * G;
    const bool valid = ii <= G_.mi - 1;
    const double v = residual_u<FAST, double, T_WRITTEN>(G_, r.u, r.v, T, r.p, r.u_ant, r.fcon, r.flin,
                                                         valid ? ii : G_.mi - 1, L0);
    if (valid) {
      r.resu[G_.at(ii, L0)] = v;
      acc += v * v;
    }
  }
  return acc;
}

// The second launch bound is the resident-CTA count a sweep at 701x301 needs
// for one wave (y-lines: one CTA per SM; x-lines: three, two with 512
// threads).  Without it ptxas held these kernels to 48-64 registers and the
// assembly issued a row's stencil loads in several rounds; with it they take
// up to 104 (y) and 85 (x) registers.
template <int EQ, int SOLVER, int TL, int G, int M>
__global__ void __launch_bounds__(TL * G, TL > 1 ? 1 : (G >= 512 ? 2 : 3))
    fused_sweep_kernel(const Geo<double> G_, const SweepIO<double> io, const SolveIO so, const int n,
                       const int line_lo, const int line_hi, const int nfull) {
  IXB_PDL_ENTRY();
  using ST = SweepTypes<SOLVER, EQ>;
  using S = typename ST::S;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* sm = reinterpret_cast<S*>(smem_raw);
  const int m = M > 0 ? M : so.m;
  const int mp = M > 0 ? (M | 1) : so.mp;
  const int L0 = 1 + blockIdx.x * TL;
  double acc_bo = 0.0;
  fused_assemble<EQ, SOLVER, TL, G, M>(sm, G_, io, m, mp, n, line_lo, line_hi, L0, acc_bo);
  __syncthreads();
  const double acc = solve_lines<S, EqIsX<EQ>::value, ST::DC, SOLVER == IXB_SOLVER_EXACT, TL, G, M>(
      sm, so, n, line_lo, line_hi, nfull, L0);
  if constexpr (EQ == EQ_TX) {
    if (so.res.resu) {
      // u residual of row jj = L0, whose T this CTA has just written (evaluating it before the
      // solve when Ri == 0, on the T the sweep reads, measured the same)
      __syncthreads();
      const double acc_res = tx_residual_row<SOLVER != IXB_SOLVER_EXACT, true, G, M>(G_, so.res, so.out, m, L0);
      const double s0 = block_sum(acc);
      const double s1 = block_sum(acc_res);
      // the energy test, then (after the loop's last pass) the outer test
      if (finish_norm2(so.nrm0, s0, so.res.ns, s1) && so.ctl.ctl && threadIdx.x == 0) {
        const bool again = ctl_inner_step(so.ctl.ctl, so.ctl.norms, so.ctl.which, so.ctl.cond);
        if (!again) ctl_outer_step(so.res.outer.ctl, so.res.outer.norms, so.res.outer.cond, so.res.outer.cond2);
      }
      return;
    }
  }
  if (io.nrm1.partials && so.nrm0.partials) {
    // p'-x: ||b_o|| and ||dp'|| with one arrival counter, then the pressure test
    const double s0 = block_sum(acc);
    const double s1 = block_sum(acc_bo);
    if (finish_norm2(so.nrm0, s0, io.nrm1, s1) && so.ctl.ctl && threadIdx.x == 0)
      ctl_inner_step(so.ctl.ctl, so.ctl.norms, so.ctl.which, so.ctl.cond);
    return;
  }
  if (io.nrm1.partials) finish_norm(io.nrm1, block_sum(acc_bo));
  if (so.nrm0.partials) {
    const bool last = finish_norm(so.nrm0, block_sum(acc));
    if (last && so.ctl.ctl && threadIdx.x == 0) ctl_inner_step(so.ctl.ctl, so.ctl.norms, so.ctl.which, so.ctl.cond);
  }
}

// Batched fused sweep: work item i = (instance, line group) of items[i]; a
// CTA walks the items grid-stride, skipping instances that no longer
// iterate; the b_o norm (p'-x) and the pass norm are reduced per instance.
template <int EQ, int SOLVER, int TL, int G>
__global__ void __launch_bounds__(TL * G)
    fused_batch_kernel(const FusedInst* __restrict__ inst, const int2* __restrict__ items, const int nitems,
                       const int* __restrict__ active, const BatchNorm bn_asm, const BatchNorm bn_sol) {
  IXB_PDL_ENTRY();
  using ST = SweepTypes<SOLVER, EQ>;
  using S = typename ST::S;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* sm = reinterpret_cast<S*>(smem_raw);
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 wi = items[it];
    if (!active[wi.x]) continue;  // uniform across the CTA
    const FusedInst& d = inst[wi.x];
    const int L0 = 1 + wi.y * TL;
    double acc_bo = 0.0;
    fused_assemble<EQ, SOLVER, TL, G, 0>(sm, d.G, d.io, d.s.io.m, d.s.io.mp, d.s.n, d.s.line_lo, d.s.line_hi, L0,
                                         acc_bo);
    __syncthreads();
    const double acc = solve_lines<S, EqIsX<EQ>::value, ST::DC, false, TL, G, 0>(sm, d.s.io, d.s.n, d.s.line_lo,
                                                                                d.s.line_hi, d.s.nfull, L0);
    if (bn_asm.partials) finish_item_norm(bn_asm, wi.x, d.s.first, d.s.count, it, block_sum(acc_bo));
    if (bn_sol.partials) finish_item_norm(bn_sol, wi.x, d.s.first, d.s.count, it, block_sum(acc));
    __syncthreads();  // the next item reuses the shared memory
  }
}

// Launch of one fused kernel; its dynamic shared-memory limit is raised the
// first time it is asked for more than before.
template <auto K>
cudaError_t fused_go(const SweepShape& s, const Geo<double>& G, const SweepIO<double>& io, const SolveIO& so,
                     cudaStream_t st) {
  // the limit is a per-device attribute of the kernel: raised once per device
  // (0: the default, 48 KB less the kernel's static shared memory)
  constexpr int kMaxDev = 64;
  static size_t limit[kMaxDev] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  if (s.smem > (limit[dev] ? limit[dev] : 48 * 1024 - 1024)) {
    e = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s.smem);
    if (e != cudaSuccess) return e;
    limit[dev] = s.smem;
  }
  if (carveout_enabled()) {
    // shared-memory carveout: just what the CTAs of one wave need per SM (one
    // y-line CTA, three x-line CTAs, two of 512 threads), the rest of the SM's
    // unified memory left to L1 for the stencil loads
    static int pct_set[kMaxDev] = {};
    int per_sm = 0;
    if ((e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess)
      return e;
    const size_t ctas = s.tl > 1 ? 1 : (s.g >= 512 ? 2 : 3);
    const size_t need = ctas * (s.smem + 1024);
    const int pct = per_sm > 0 ? (int)std::min<size_t>(100, (need * 100 + per_sm - 1) / per_sm) : 100;
    if (pct != pct_set[dev]) {
      if ((e = cudaFuncSetAttribute(K, cudaFuncAttributePreferredSharedMemoryCarveout, pct)) != cudaSuccess) return e;
      pct_set[dev] = pct;
    }
  }
  return launch_k(K, s.grid, s.tl * s.g, s.smem, st, G, io, so, s.n, s.line_lo, s.line_hi, s.nfull);
}

// Launches the fused form of sweep EQ for the shapes of IXB_FUSED_X_SHAPES /
// IXB_FUSED_Y_SHAPES; any other shape: cudaErrorNotSupported (the caller
// runs the two-kernel sweep).
template <int EQ, int SOLVER>
cudaError_t fused_launch(const SweepShape& s, const Geo<double>& G, const SweepIO<double>& io, const SolveIO& so,
                         cudaStream_t st) {
  constexpr bool EXACT = SOLVER == IXB_SOLVER_EXACT;
#define IXB_FUSED_(TL_, G_)                                                                     \
  if (s.tl == TL_ && s.g == G_) {                                                               \
    if (!EXACT && s.m == 3) return fused_go<fused_sweep_kernel<EQ, SOLVER, TL_, G_, 3>>(s, G, io, so, st); \
    if constexpr (!EqIsX<EQ>::value && !EXACT)                                                  \
      if (s.m == 5) return fused_go<fused_sweep_kernel<EQ, SOLVER, TL_, G_, 5>>(s, G, io, so, st); \
    return fused_go<fused_sweep_kernel<EQ, SOLVER, TL_, G_, 0>>(s, G, io, so, st);                \
  }
  if constexpr (EqIsX<EQ>::value) {
    IXB_FUSED_X_SHAPES(IXB_FUSED_)
  } else {
    IXB_FUSED_Y_SHAPES(IXB_FUSED_)
  }
#undef IXB_FUSED_
  return cudaErrorNotSupported;
}

// Launches the batched fused form of sweep EQ with one shape (TL x G) for
// every instance; cudaErrorNotSupported for shapes outside IXB_FUSED_*_SHAPES.
template <int EQ, int SOLVER>
cudaError_t fused_batch_launch(int tl, int g, size_t smem, const FusedInst* inst, const int2* items, int nitems,
                               const int* active, const BatchNorm& bn_asm, const BatchNorm& bn_sol,
                               cudaStream_t st) {
  auto go = [&](auto k, int nt) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0, dev = 0, nsm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, nt, smem)) != cudaSuccess) return e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidValue;
    const int grid = std::max(1, std::min(nitems, per_sm * nsm));
    return launch_k(k, grid, nt, smem, st, inst, items, nitems, active, bn_asm, bn_sol);
  };
#define IXB_FBATCH_(TL_, G_) \
  if (tl == TL_ && g == G_) return go(fused_batch_kernel<EQ, SOLVER, TL_, G_>, TL_ * G_);
  if constexpr (EqIsX<EQ>::value) {
    IXB_FUSED_X_SHAPES(IXB_FBATCH_)
  } else {
    IXB_FUSED_Y_SHAPES(IXB_FBATCH_)
  }
#undef IXB_FBATCH_
  return cudaErrorNotSupported;
}

}  // namespace ixb
