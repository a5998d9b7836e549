// ixb_sweep.cuh -- the fused line-sweep kernel (assembly + boundary rows +
// partitioned line solve + write-back with the pass norm), included by the
// per-equation translation units ixb_sweep_{u,v,p,t}.cu.
//
// One fused kernel per line sweep replaces the reference's four OpenACC
// regions per sweep (assembly, impone_cond_frontera, tridiagonal, scatter;
// e.g. source/main.f90:420-484): a CTA owns TL adjacent lines, assembles
// their rows straight from the fields into shared memory (coalesced along
// ii), applies the boundary rows from a per-line table, solves the lines with
// G = 256/TL threads each, and writes the solution to the ping-pong output
// buffer, reducing the convergence norm of the pass on the way out.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "ixb_internal.h"
#include "ixb_reduce.cuh"

namespace ixb {

// ---------------------------------------------------------------------------
// per-equation assembly dispatch
// ---------------------------------------------------------------------------
template <int EQ>
struct EqIsX { static constexpr bool value = (EQ & 1) != 0; };

template <class R, int EQ, bool FAST, class F>
__device__ __forceinline__ Row<R> assemble_cell(const Geo<R>& G, const SweepIO<F>& io, int ii, int jj,
                                                double& acc_bo) {
  if constexpr (EQ == EQ_UY) {
    return assemble_uy<FAST>(G, io, ii, jj);
  } else if constexpr (EQ == EQ_UX) {
    R au;
    Row<R> r = assemble_ux<FAST>(G, io, ii, jj, au);
    io.aux[G.at(ii, jj)] = F(au);
    return r;
  } else if constexpr (EQ == EQ_VY) {
    return assemble_vy<FAST>(G, io, ii, jj);
  } else if constexpr (EQ == EQ_VX) {
    R av;
    Row<R> r = assemble_vx<FAST>(G, io, ii, jj, av);
    io.aux[G.at(ii, jj)] = F(av);
    return r;
  } else if constexpr (EQ == EQ_PY) {
    return assemble_py<FAST>(G, io, ii, jj);
  } else if constexpr (EQ == EQ_PX) {
    F bo;
    Row<R> r = assemble_px<FAST>(G, io, ii, jj, bo);
    io.aux[G.at(ii, jj)] = bo;
    acc_bo += (double)bo * (double)bo;
    return r;
  } else if constexpr (EQ == EQ_TY) {
    return assemble_ty<FAST>(G, io, ii, jj);
  } else {
    return assemble_tx<FAST>(G, io, ii, jj);
  }
}

// Arithmetic types of one sweep.  The binary64 solvers use binary64
// throughout.  The mixed solver (handle precision IXB_PREC_FP32_REFINED)
// stages and solves every line in binary32.  The u, v and T rows are
// assembled in binary64 and turned into a defect correction (DC): the
// binary64 residual d - A x of the current values is solved for in binary32
// and the correction added back in binary64, so the fixed point of these
// equations is the binary64 one.  The p' rows are assembled and solved in
// binary32 (p' only steers the iteration; it vanishes at convergence), with
// their mass source b_o evaluated in binary64.
template <int SOLVER, int EQ>
struct SweepTypes {
  static constexpr bool MIX = SOLVER == SOLVER_MIXED;
  static constexpr bool DC = MIX && EQ != EQ_PY && EQ != EQ_PX;
  using S = typename std::conditional<MIX, float, double>::type;        // staged rows, line solve
  using A = typename std::conditional<MIX && !DC, float, double>::type;  // coefficient assembly
};

template <class A>
__host__ __device__ inline const Geo<A>& pick_geo(const Geo<double>& d, const Geo<float>& f) {
  if constexpr (std::is_same<A, float>::value) return f; else return d;
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
// fused sweep kernel: TL lines per CTA, G threads per line (TL*G = 256)
// ---------------------------------------------------------------------------
template <class R, int EQ, int SOLVER, int TL, int G, int M>
__global__ void __launch_bounds__(TL * G)
    sweep_kernel(const Geo<typename SweepTypes<SOLVER, EQ>::A> G_, const SweepIO<R> io, const int n,
                 const int line_lo, const int line_hi, const int nfull) {
  using ST = SweepTypes<SOLVER, EQ>;
  using S = typename ST::S;
  using A = typename ST::A;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* sm = reinterpret_cast<S*>(smem_raw);
  constexpr bool X = EqIsX<EQ>::value;
  constexpr int NT = TL * G;
  const Geo<A>& Gm = G_;
  // M > 0: chunk length known at compile time (divisions by it become
  // multiply-shifts and the per-thread loops unroll)
  const int m = M > 0 ? M : io.m;
  const int mp = M > 0 ? (M | 1) : io.mp;
  const int npad = G * m;
  const int LS = (int)line_smem_elems(G, mp);
  const int arr = G * mp;
  const int L0 = 1 + blockIdx.x * TL;
  double acc_bo = 0.0;

  // phase 1: assemble every row of the solved lines into shared memory;
  // TL*npad = NT*m, so every thread handles exactly m rows
#pragma unroll
  for (int it = 0; it < (M > 0 ? M : 32); ++it) {  // m <= 25 (ixb_create bounds the grid)
    if (M == 0 && it >= m) break;
    const int idx = threadIdx.x + it * NT;
    int l, r;
    if (X) { l = TL == 1 ? 0 : idx / npad; r = idx - l * npad; }
    else { l = idx % TL; r = idx / TL; }
    const int L = L0 + l;
    if (L < line_lo || L > line_hi) continue;
    Row<A> row;
    if (r >= n) row = Row<A>{A(0), A(1), A(0), A(0)};  // identity padding
    else if (r == 0) row = bc_first_row<A>(io.bc_first, L);
    else if (r == n - 1) row = bc_last_row<A>(io.bc_last, L);
    else {
      const int ii = X ? r + 1 : L;
      const int jj = X ? L : r + 1;
      row = assemble_cell<A, EQ, SOLVER != IXB_SOLVER_EXACT>(Gm, io, ii, jj, acc_bo);
    }
    if constexpr (ST::DC) {
      // defect correction: the row's binary64 residual at the current values
      if (r < n) {
        const int g = Gm.at(X ? r + 1 : L, X ? L : r + 1);
        const int step = X ? 1 : Gm.LD;
        double res = fma(-row.b, __ldg(io.in + g), row.d);
        if (r > 0) res = fma(-row.a, __ldg(io.in + g - step), res);
        if (r < n - 1) res = fma(-row.c, __ldg(io.in + g + step), res);
        row.d = res;
      }
    }
    const int ch = r / m;
    const int o = l * LS + ch * mp + (r - ch * m);
    sm[o] = S(row.a);
    sm[o + arr] = S(row.b);
    sm[o + 2 * arr] = S(row.c);
    sm[o + 3 * arr] = S(row.d);
  }
  __syncthreads();

  // phase 2: line solves
  {
    const int l = threadIdx.x / G;
    const int L = L0 + l;
    const bool active = (L >= line_lo && L <= line_hi);
    S* line = sm + l * LS;
    if constexpr (SOLVER == IXB_SOLVER_EXACT) {
      if (active && threadIdx.x % G == 0) thomas_exact(line, line + arr, line + 2 * arr, line + 3 * arr, n, m, mp);
    } else {
      chunk_solve<S, G>(line, m, mp, active, RS_PCR);
    }
  }
  __syncthreads();

  // phase 3: write the new field (unsolved lines keep their values) and
  // accumulate ||new - prev|| over the interior rows of the solved lines
  double acc = 0.0;
  for (int idx = threadIdx.x; idx < TL * n; idx += NT) {
    int l, r;
    if (X) { l = TL == 1 ? 0 : idx / n; r = idx - l * n; }
    else { l = idx % TL; r = idx / TL; }
    const int L = L0 + l;
    if (L > nfull) continue;
    const int ii = X ? r + 1 : L;
    const int jj = X ? L : r + 1;
    const int g = Gm.at(ii, jj);
    R x;
    if (L >= line_lo && L <= line_hi) {
      const int ch = r / m;
      const S xs = sm[l * LS + 3 * arr + ch * mp + (r - ch * m)];
      if constexpr (ST::DC) x = io.in[g] + R(xs);
      else x = R(xs);
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


// Launch shapes (lines per CTA x threads per line); 128 or 256 threads.
#define IXB_SWEEP_SHAPES(X_) X_(1, 128) X_(1, 256) X_(2, 64) X_(2, 128) X_(4, 32) X_(4, 64) X_(8, 32)

template <class R, int EQ, int SOLVER, int TL, int G>
static cudaError_t sweep_launch_one(const SweepShape& s, const Geo<double>& Gd, const Geo<float>& Gf,
                                    const SweepIO<R>& io, cudaStream_t st) {
  const auto& Gm = pick_geo<typename SweepTypes<SOLVER, EQ>::A>(Gd, Gf);
  if (SOLVER != IXB_SOLVER_EXACT && s.m == 3) {
    sweep_kernel<R, EQ, SOLVER, TL, G, 3><<<s.grid, TL * G, s.smem, st>>>(Gm, io, s.n, s.line_lo, s.line_hi, s.nfull);
  } else {
    sweep_kernel<R, EQ, SOLVER, TL, G, 0><<<s.grid, TL * G, s.smem, st>>>(Gm, io, s.n, s.line_lo, s.line_hi, s.nfull);
  }
  return cudaGetLastError();
}

template <class R, int EQ, int SOLVER>
cudaError_t sweep_launch_solver(const SweepShape& s, const Geo<double>& Gd, const Geo<float>& Gf,
                                const SweepIO<R>& io, cudaStream_t st) {
#define IXB_CASE_(TL_, G_) \
  if (s.tl == TL_ && s.g == G_) return sweep_launch_one<R, EQ, SOLVER, TL_, G_>(s, Gd, Gf, io, st);
  IXB_SWEEP_SHAPES(IXB_CASE_)
#undef IXB_CASE_
  return cudaErrorInvalidValue;
}

template <class R, int EQ, int SOLVER>
cudaError_t sweep_smem_limit_solver(int bytes) {
  cudaError_t e = cudaSuccess;
  auto set = [&](auto k) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  };
#define IXB_SET_(TL_, G_)                        \
  if (SOLVER != IXB_SOLVER_EXACT)              \
    set(sweep_kernel<R, EQ, SOLVER, TL_, G_, 3>); \
  set(sweep_kernel<R, EQ, SOLVER, TL_, G_, 0>);
  IXB_SWEEP_SHAPES(IXB_SET_)
#undef IXB_SET_
  return e;
}

// Resident CTAs per SM of the kernel a shape launches (0 if it cannot run).
template <class R, int EQ, int SOLVER>
int sweep_blocks_per_sm_solver(const SweepShape& s) {
  int nb = 0;
  cudaError_t e = cudaErrorInvalidValue;
#define IXB_OCC_(TL_, G_)                                                                                    \
  if (s.tl == TL_ && s.g == G_) {                                                                            \
    if (SOLVER != IXB_SOLVER_EXACT && s.m == 3)                                                              \
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, sweep_kernel<R, EQ, SOLVER, TL_, G_, 3>,         \
                                                        TL_ * G_, s.smem);                                   \
    else                                                                                                     \
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, sweep_kernel<R, EQ, SOLVER, TL_, G_, 0>,         \
                                                        TL_ * G_, s.smem);                                   \
  }
  IXB_SWEEP_SHAPES(IXB_OCC_)
#undef IXB_OCC_
  return e == cudaSuccess ? nb : 0;
}

}  // namespace ixb
