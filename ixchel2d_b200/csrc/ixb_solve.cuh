// ixb_solve.cuh -- the in-shared-memory half of a line solve, shared by the
// staged line-solve kernels (ixb_solve.cu) and the fused x-sweep kernels
// (ixb_sweep.cuh): TL lines already in shared memory in the chunk layout of
// chunk_solve are solved and written to the field's output buffer.
#pragma once
#include <cuda_runtime.h>

#include "ixb_internal.h"

namespace ixb {

// Lines L0 .. L0+TL-1 of one sweep, rows in shared memory (line l at
// sm + l * line_smem_elems(G, mp), arrays a | b | c | d of G chunks of m
// rows at pitch mp): solve, then write the new field (lines outside
// line_lo..line_hi keep their values) and return this thread's share of
// ||new - prev||^2 over the interior rows of the solved lines.  y-lines are
// written TL adjacent ii at a time.  Called by all threads of the CTA (it
// holds barriers).
template <class S, bool X, bool DC, bool EXACT, int TL, int G, int M>
__device__ __forceinline__ double solve_lines(S* sm, const SolveIO& io, const int n, const int line_lo,
                                              const int line_hi, const int nfull, const int L0) {
  constexpr int NT = TL * G;
  const int m = M > 0 ? M : io.m;
  const int mp = M > 0 ? (M | 1) : io.mp;
  const int LS = (int)line_smem_elems(G, mp);
  const int arr = G * mp;
  {
    const int l = threadIdx.x / G;
    const int L = L0 + l;
    const bool active = (L >= line_lo && L <= line_hi);
    S* line = sm + l * LS;
    if constexpr (EXACT) {
      if (active && threadIdx.x % G == 0) thomas_exact(line, line + arr, line + 2 * arr, line + 3 * arr, n, m, mp);
    } else {
      chunk_solve<S, G, TL>(line, m, mp, active, RS_PCR);
    }
  }
  __syncthreads();
  double acc = 0.0;
  for (int idx = threadIdx.x; idx < TL * n; idx += NT) {
    int l, r;
    if (X) { l = TL == 1 ? 0 : idx / n; r = idx - l * n; }
    else { l = idx % TL; r = idx / TL; }
    const int L = L0 + l;
    if (L > nfull) continue;
    const int g = X ? (L - 1) * io.LD + r : r * io.LD + (L - 1);
    double x;
    if (L >= line_lo && L <= line_hi) {
      const int ch = r / m;
      const S xs = sm[l * LS + 3 * arr + ch * mp + (r - ch * m)];
      if constexpr (DC) x = io.in[g] + double(xs);
      else x = double(xs);
      if (r >= 1 && r <= n - 2) {
        const double dv = x - (io.prev ? io.prev[g] : 0.0);
        acc += dv * dv;
      }
    } else {
      x = io.in[g];
    }
    io.out[g] = x;
  }
  return acc;
}

}  // namespace ixb
