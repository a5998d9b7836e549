// ixb_adjoint_fast.cu -- discrete adjoint of the energy iteration with the
// flow held fixed: the gradient of the hot-wall Nusselt number after K
// passes of the T sweeps (T-y then T-x, source/main.f90:985-1136) with
// respect to the Dirichlet value of every x-line on side a (the hot wall,
// x = 0).  The reference has no counterpart.
//
// With u, v frozen, every T sweep is affine in the temperatures: a line solve
// x = A^-1 (R T_in + f) with coefficients (AI, AD, BS, BN and the relaxed
// diagonal) that depend on the mesh and the velocities only, and f holding
// the boundary values.  The adjoint therefore needs no stored forward states:
// starting from the Nusselt number's weights, each sweep is reversed as
// mu = A^-T lambda (a transposed batched line solve) followed by
// lambda_in = R^T mu plus the lines the sweep copies, and the side-a
// boundary rows of the x-sweeps collect d Nu / d value += mu[row 0].
// Built with FMA contraction, like the fast forward assembly, whose
// coefficients it re-evaluates.  ixb_adjoint_energy_coupled extends this to
// K outer SIMPLE iterations of a flow that evolves but does not depend on
// the temperature, with checkpoints every C iterations.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <functional>
#include <vector>

#include "ixb_handle.h"
#include "ixb_nusselt.h"

namespace ixb {
namespace {

// coefficient arrays (field layout) of the energy rows: AI, AD, BS, BN, diag
enum { C_AI = 0, C_AD, C_BS, C_BN, C_DG, C_COUNT };

__global__ void adj_coef_kernel(const Geo<double> G, const SweepIO<double> io, double* __restrict__ coef,
                                size_t fsz) {
  const int ni = G.mi - 1;  // ii = 2..mi, jj = 2..nj
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ni * (G.nj - 1)) return;
  const int ii = 2 + idx % ni, jj = 2 + idx / ni;
  const Row<double> rx = assemble_tx<true>(G, io, ii, jj);  // a = AI, c = AD, b = diagonal
  const Row<double> ry = assemble_ty<true>(G, io, ii, jj);  // a = BS, c = BN
  const int c0 = G.at(ii, jj);
  coef[C_AI * fsz + c0] = rx.a;
  coef[C_AD * fsz + c0] = rx.c;
  coef[C_BS * fsz + c0] = ry.a;
  coef[C_BN * fsz + c0] = ry.c;
  coef[C_DG * fsz + c0] = rx.b;
}

struct Sweep {
  bool x;               // x-lines (fixed jj) or y-lines (fixed ii)
  int n;                // rows per line
  int nl;               // solved lines 2 .. nl+1
  const BCEntry* first;
  const BCEntry* last;
};

// Forward row r of solved line L: (a, b, c) of impone_cond_frontera's boundary
// rows or of the energy assembly.
__device__ __forceinline__ void fwd_row(const Geo<double>& G, const Sweep& s, const double* coef, size_t fsz, int L,
                                        int r, double& a, double& b, double& c) {
  if (r == 0) {
    const BCEntry e = s.first[L];
    a = 0.0; b = e.type == 2 ? -1.0 : 1.0; c = e.type == 2 ? 1.0 : 0.0;
  } else if (r == s.n - 1) {
    const BCEntry e = s.last[L];
    a = e.type == 2 ? -1.0 : 0.0; b = 1.0; c = 0.0;
  } else {
    const int c0 = s.x ? G.at(r + 1, L) : G.at(L, r + 1);
    a = coef[(s.x ? C_AI : C_BS) * fsz + c0];
    c = coef[(s.x ? C_AD : C_BN) * fsz + c0];
    b = coef[C_DG * fsz + c0];
  }
}

// Transposed rows (a'_r = c_{r-1}, b'_r = b_r, c'_r = a_{r+1}) and right-hand
// side lambda of every solved line, contiguous per line.
__global__ void adj_stage_kernel(const Geo<double> G, const Sweep s, const double* __restrict__ coef, size_t fsz,
                                 const double* __restrict__ lam, double* __restrict__ ta, double* __restrict__ tb,
                                 double* __restrict__ tc, double* __restrict__ td) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= s.nl * s.n) return;
  const int li = idx / s.n, r = idx - li * s.n, L = li + 2;
  double a, b, c, t;
  fwd_row(G, s, coef, fsz, L, r, a, b, c);
  ta[idx] = 0.0;
  tc[idx] = 0.0;
  if (r > 0) { fwd_row(G, s, coef, fsz, L, r - 1, t, t, c); ta[idx] = c; }
  if (r < s.n - 1) { fwd_row(G, s, coef, fsz, L, r + 1, a, t, t); tc[idx] = a; }
  fwd_row(G, s, coef, fsz, L, r, a, b, c);
  tb[idx] = b;
  td[idx] = lam[s.x ? G.at(r + 1, L) : G.at(L, r + 1)];
}

// lambda_in = R^T mu + copies of the unsolved lines; x-sweeps also add the
// side-a boundary rows' sensitivities to grad (indexed by line).
__global__ void adj_scatter_kernel(const Geo<double> G, const Sweep s, const double* __restrict__ coef, size_t fsz,
                                   double rel, const double* __restrict__ mu, const double* __restrict__ lam_out,
                                   double* __restrict__ lam_in, double* __restrict__ grad) {
  const int nx = G.mi + 1, ny = G.nj + 1;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nx * ny) return;
  const int ii = 1 + idx % nx, jj = 1 + idx / nx;
  const int L = s.x ? jj : ii;  // line of this cell
  const int r = s.x ? ii - 1 : jj - 1;
  const int nfull = s.nl + 2;
  auto solved = [&](int l) { return l >= 2 && l <= s.nl + 1; };
  auto mu_at = [&](int l, int rr) { return mu[(size_t)(l - 2) * s.n + rr]; };
  const bool interior = r >= 1 && r <= s.n - 2;
  double v = 0.0;
  if (L >= 1 && L <= nfull) {
    if (solved(L)) {
      if (interior) v += coef[C_DG * fsz + G.at(ii, jj)] * (1.0 - rel) * mu_at(L, r);
      if (s.x && r == 0) grad[L] += mu_at(L, 0);
    } else {
      v += lam_out[G.at(ii, jj)];
    }
    // rows of the neighbouring lines that read this cell through d
    if (interior) {
      if (solved(L + 1)) {
        const int cn = s.x ? G.at(ii, jj + 1) : G.at(ii + 1, jj);
        v -= coef[(s.x ? C_BS : C_AI) * fsz + cn] * mu_at(L + 1, r);
      }
      if (solved(L - 1)) {
        const int cp = s.x ? G.at(ii, jj - 1) : G.at(ii - 1, jj);
        v -= coef[(s.x ? C_BN : C_AD) * fsz + cp] * mu_at(L - 1, r);
      }
    }
  }
  lam_in[G.at(ii, jj)] = v;
}

}  // namespace
}  // namespace ixb

using namespace ixb;

#define ACK(x)                   \
  do {                           \
    cudaError_t e_ = (x);        \
    if (e_ != cudaSuccess) {     \
      h->last_cuda = e_;         \
      return IXB_ECUDA;          \
    }                            \
  } while (0)
#define TRY(x)                   \
  do {                           \
    const int s_ = (x);          \
    if (s_ != IXB_OK) return s_; \
  } while (0)

namespace {

// Workspace, objective weights and reversed (T-y, T-x) passes shared by the
// two adjoint entry points.
struct AdjCtx {
  ixb_handle* h;
  size_t fsz = 0;
  double *coef = nullptr, *lam = nullptr, *lam2 = nullptr, *ta = nullptr, *tb = nullptr, *tc = nullptr,
         *td = nullptr, *mu = nullptr, *gd = nullptr;
  Geo<double> G{};
  Sweep sx{}, sy{};
  double rel = 0.0;
  int cells = 0;

  int init(int j0, int j1) {
    const int mi = h->mi, nj = h->nj;
    fsz = h->fsz;
    const size_t nst = (size_t)std::max((nj - 1) * (mi + 1), (mi - 1) * (nj + 1));
    const size_t need = (C_COUNT + 2) * fsz + 5 * nst + (size_t)(nj + 2);
    if (h->adj_size < need) {
      if (h->adj_pool) cudaFree(h->adj_pool);
      h->adj_pool = nullptr;
      h->adj_size = 0;
      ACK(cudaMalloc(&h->adj_pool, need * sizeof(double)));
      h->adj_size = need;
    }
    coef = h->adj_pool;
    lam = coef + C_COUNT * fsz;
    lam2 = lam + fsz;
    ta = lam2 + fsz;
    tb = ta + nst;
    tc = tb + nst;
    td = tc + nst;
    mu = td + nst;
    gd = mu + nst;
    G = handle_geo(h);
    const BCEntry* base = h->bc + (size_t)2 * 4 * h->bcstride;  // T tables, sides a b c d
    sx = Sweep{true, mi + 1, nj - 1, base + 0 * (size_t)h->bcstride, base + 2 * (size_t)h->bcstride};
    sy = Sweep{false, nj + 1, mi - 1, base + 1 * (size_t)h->bcstride, base + 3 * (size_t)h->bcstride};
    rel = h->prm.rel_ener;
    cells = (mi + 1) * (nj + 1);
    // the objective's weights: Nu is linear in T (the wall-normal 3-point
    // derivative integrated panel by panel), evaluated here on unit fields
    std::vector<double> along(nj + 2, 0.0), across(mi + 2, 0.0);
    for (int j = 1; j <= nj + 1; ++j) along[j] = h->yp[j - 1];
    for (int i = 1; i <= mi + 1; ++i) across[i] = h->xp[i - 1];
    std::vector<double> w((size_t)fsz, 0.0);
    for (int k = j0; k <= j1 + 2; ++k)
      for (int l = 1; l <= 3; ++l) {
        auto f = [&](int kk, int ll) { return (kk == k && ll == l) ? 1.0 : 0.0; };
        w[(size_t)(k - 1) * h->LD + (l - 1)] = nusselt_wall(f, along.data(), across.data(), mi + 1, 0, 0, j0, j1);
      }
    ACK(cudaMemcpyAsync(lam, w.data(), fsz * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    ACK(cudaMemsetAsync(gd, 0, (nj + 2) * sizeof(double), h->stream));
    ACK(cudaStreamSynchronize(h->stream));  // w leaves scope
    return IXB_OK;
  }

  // coefficients of the energy rows at the handle's current velocities
  int coefficients() {
    const int cT = h->cT;
    SweepIO<double> io = handle_sweep_io(h, EQ_TX, nullptr);
    h->cT = cT;
    ACK(cudaMemsetAsync(coef, 0, C_COUNT * fsz * sizeof(double), h->stream));
    const int n = (h->mi - 1) * (h->nj - 1);
    adj_coef_kernel<<<(n + 255) / 256, 256, 0, h->stream>>>(G, io, coef, fsz);
    ACK(cudaGetLastError());
    return IXB_OK;
  }

  int reverse(const Sweep& s, const double* lam_out, double* lam_in) {
    const int rows = s.nl * s.n;
    adj_stage_kernel<<<(rows + 255) / 256, 256, 0, h->stream>>>(G, s, coef, fsz, lam_out, ta, tb, tc, td);
    ACK(cudaGetLastError());
    ACK(tridiag_f64(ta, tb, tc, td, mu, s.n, s.nl, 0, IXB_SOLVER_HYBRID, h->stream));
    adj_scatter_kernel<<<(cells + 255) / 256, 256, 0, h->stream>>>(G, s, coef, fsz, rel, mu, lam_out, lam_in, gd);
    ACK(cudaGetLastError());
    return IXB_OK;
  }

  // one (T-y, T-x) pass, reversed: T-x first
  int pass() {
    const int r1 = reverse(sx, lam, lam2);
    return r1 != IXB_OK ? r1 : reverse(sy, lam2, lam);
  }

  int finish(double* grad) {
    const int nj = h->nj;
    std::vector<double> g(nj + 2);
    ACK(cudaMemcpyAsync(g.data(), gd, (nj + 2) * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    ACK(cudaStreamSynchronize(h->stream));
    int timed_out = 0;
    ACK(tridiag_take_timeout(&timed_out));  // a line solve whose copies did not arrive in time
    if (timed_out) return IXB_ETIMEOUT;
    for (int jj = 1; jj <= nj + 1; ++jj) grad[jj - 1] = g[jj];
    return IXB_OK;
  }
};

int check_range(const ixb_handle* h, int j0, int j1) {
  if (j0 < 1 || j1 < j0) return IXB_EINVAL;
  for (int k = j0; k <= j1; k += 2)
    if (k + 2 > h->nj + 1) return IXB_EINVAL;
  return IXB_OK;
}

}  // namespace

extern "C" int ixb_adjoint_energy(ixb_handle* h, int K, int j0, int j1, double* grad) {
  if (!h || K < 0 || !grad) return IXB_EINVAL;
  const int st0 = handle_ready(h);
  if (st0 != IXB_OK) return st0;
  TRY(check_range(h, j0, j1));
  AdjCtx A{h};
  TRY(A.init(j0, j1));
  TRY(A.coefficients());  // the frozen velocities
  // K passes of (T-y, T-x), reversed.  A WHILE graph runs them kLoopUnroll
  // at a time (rebuilt when the handle or its workspace changes); the
  // remaining K mod kLoopUnroll are plain launches
  const std::function<int()> pass = [&A]() -> int { return A.pass(); };
  if (K >= kLoopUnroll) {
    if (h->agraph_dirty || !h->agraph_exec || h->agraph_pool != h->adj_pool) {
      const int r = handle_build_loop_graph(h, pass, kLoopUnroll, &h->agraph, &h->agraph_exec);
      if (r != IXB_OK) return r;
      h->agraph_dirty = false;
      h->agraph_pool = h->adj_pool;
    }
    const int r = handle_run_loop_graph(h, h->agraph_exec, K / kLoopUnroll);
    if (r != IXB_OK) return r;
  }
  for (int k = 0; k < K % kLoopUnroll; ++k) TRY(pass());
  return A.finish(grad);
}

// The energy adjoint through K outer SIMPLE iterations whose flow evolves
// but does not depend on the temperature (Ri = Riy = 0: the buoyancy terms
// are exact zeros, so the velocities of every iteration are the same for
// any wall temperature).  T after K iterations is then a composition of
// affine T passes, the passes of iteration k with the coefficients of that
// iteration's velocities, and the gradient is exact.  Forward: K single
// outer iterations, recording each one's T passes and checkpointing the
// seven state fields every C iterations.  Reverse, segment by segment:
// restore the segment's checkpoint, recompute it storing u, v after every
// iteration, then reverse its iterations' T passes with their coefficients.
extern "C" int ixb_adjoint_energy_coupled(ixb_handle* h, int K, int C, int j0, int j1, double* grad,
                                          double* nu0) {
  if (!h || K < 1 || C < 1 || !grad) return IXB_EINVAL;
  const int st0 = handle_ready(h);
  if (st0 != IXB_OK) return st0;
  TRY(check_range(h, j0, j1));
  if (h->prm.Ri != 0.0 || h->prm.Riy != 0.0) return IXB_EINVAL;  // the flow would depend on T
  if (C > K) C = K;
  const size_t fsz = h->fsz, fb = fsz * sizeof(double);
  const int nseg = (K + C - 1) / C;
  // checkpoints: u v p T u_ant v_ant T_ant at iterations 0, C, 2C, ... and K
  double* pool = nullptr;
  const size_t ncp = (size_t)nseg + 1;
  ACK(cudaMalloc(&pool, (ncp * 7 + (size_t)2 * C) * fb));
  double* useg = pool + ncp * 7 * fsz;  // u after each iteration of a segment
  double* vseg = useg + (size_t)C * fsz;
  struct Saved { int iter_ecuaci, iter_simple; };
  std::vector<Saved> counters(ncp);
  auto fields = [h]() {
    return std::array<double*, 7>{h->u[h->cu], h->v[h->cv], h->p, h->T[h->cT], h->u_ant, h->v_ant, h->T_ant};
  };
  auto save = [&](size_t slot) -> int {
    const auto f = fields();
    for (int k = 0; k < 7; ++k)
      ACK(cudaMemcpyAsync(pool + (slot * 7 + k) * fsz, f[k], fb, cudaMemcpyDeviceToDevice, h->stream));
    counters[slot] = Saved{h->iter_ecuaci, h->iter_simple};
    return IXB_OK;
  };
  auto restore = [&](size_t slot) -> int {
    const auto f = fields();
    for (int k = 0; k < 7; ++k)
      ACK(cudaMemcpyAsync(f[k], pool + (slot * 7 + k) * fsz, fb, cudaMemcpyDeviceToDevice, h->stream));
    h->iter_ecuaci = counters[slot].iter_ecuaci;
    h->iter_simple = counters[slot].iter_simple;
    return IXB_OK;
  };
  int st = IXB_OK;
  std::vector<int> passes(K + 1, 0);  // T passes of iteration k
  auto run = [&]() -> int {
    // forward: K iterations, one call each (their T pass counts)
    TRY(save(0));
    for (int k = 1; k <= K; ++k) {
      ixb_report rep{};
      TRY(ixb_simple_iterations(h, 1, &rep));
      passes[k] = (int)rep.n_ener;
      if (k % C == 0 && k < K) TRY(save((size_t)(k / C)));
    }
    TRY(save(ncp - 1));  // the final state, restored at the end
    if (nu0) TRY(ixb_nusselt_x(h, j0, j1, nu0, nullptr));
    AdjCtx A{h};
    TRY(A.init(j0, j1));
    for (int seg = nseg - 1; seg >= 0; --seg) {
      const int k0 = seg * C, k1 = std::min(K, k0 + C);  // iterations k0+1 .. k1
      TRY(restore((size_t)seg));
      for (int k = k0 + 1; k <= k1; ++k) {
        ixb_report rep{};
        TRY(ixb_simple_iterations(h, 1, &rep));
        if ((int)rep.n_ener != passes[k]) return IXB_ESTATE;  // the recomputation must retrace the forward
        ACK(cudaMemcpyAsync(useg + (size_t)(k - k0 - 1) * fsz, h->u[h->cu], fb, cudaMemcpyDeviceToDevice, h->stream));
        ACK(cudaMemcpyAsync(vseg + (size_t)(k - k0 - 1) * fsz, h->v[h->cv], fb, cudaMemcpyDeviceToDevice, h->stream));
      }
      for (int k = k1; k > k0; --k) {
        ACK(cudaMemcpyAsync(h->u[h->cu], useg + (size_t)(k - k0 - 1) * fsz, fb, cudaMemcpyDeviceToDevice, h->stream));
        ACK(cudaMemcpyAsync(h->v[h->cv], vseg + (size_t)(k - k0 - 1) * fsz, fb, cudaMemcpyDeviceToDevice, h->stream));
        TRY(A.coefficients());
        for (int q = 0; q < passes[k]; ++q) TRY(A.pass());
      }
    }
    TRY(restore(ncp - 1));
    return A.finish(grad);
  };
  st = run();
  cudaStreamSynchronize(h->stream);
  cudaFree(pool);
  return st;
}
