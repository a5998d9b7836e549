// ixb_api.cu -- the C ABI of include/ixb.h: handle lifetime, state transfer,
// boundary tables and the SIMPLE driver loop on one CUDA stream.
//
// The outer iteration (source/main.f90:395-1217) runs as one CUDA graph per
// handle: the reference's three inner loops and the outer loop are WHILE
// conditional nodes whose conditions are set on the device by the kernels
// that finish each norm, applying the reference's exit tests, so a whole
// SIMPLE loop is one graph launch with no host round trip.  Fixed counts
// that are multiples of four use a second graph with four outer passes per
// WHILE body.  The same sequence can also be driven from the host (one sync
// per inner pass) for debugging.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "ixb_ctl.cuh"
#include "ixb_handle.h"

using namespace ixb;

namespace {

#define CK(x)                                    \
  do {                                           \
    cudaError_t e_ = (x);                        \
    if (e_ != cudaSuccess) {                     \
      h->last_cuda = e_;                         \
      return IXB_ECUDA;                          \
    }                                            \
  } while (0)

}  // namespace


namespace {

Geo<double> make_geo(const ixb_handle* h) {
  Geo<double> G{};
  G.mi = h->mi; G.nj = h->nj; G.LD = h->LD; G.mstride = h->mstride; G.m = h->metrics;
  G.tstride = h->fsz; G.tab = h->tables;
  G.gm = h->prm.gamma_momen; G.ge = h->prm.gamma_energ; G.Ri = h->prm.Ri; G.Riy = h->prm.Riy;
  G.dt = h->prm.dt; G.rel_vel = h->prm.rel_vel; G.rel_pres = h->prm.rel_pres; G.rel_ener = h->prm.rel_ener;
  G.p_update = h->prm.p_update;
  G.inv_gm = 1.0 / G.gm; G.inv_dt = 1.0 / G.dt; G.inv_rel_vel = 1.0 / G.rel_vel;
  G.inv_rel_pres = 1.0 / G.rel_pres; G.inv_rel_ener = 1.0 / G.rel_ener;
  return G;
}

// line-solve form of the sweeps: the handle's precision picks the mixed form
// in place of the binary64 hybrid one
int solver_form(const ixb_handle* h) {
  return (h->prec == IXB_PREC_FP32_REFINED && h->prm.solver == IXB_SOLVER_HYBRID) ? SOLVER_MIXED : h->prm.solver;
}
int real_bytes(const ixb_handle* h) { return solver_form(h) == SOLVER_MIXED ? 4 : 8; }

NormSlot slot(ixb_handle* h, int k) {
  return NormSlot{h->partials + (size_t)k * h->pstride, h->counters + k, h->norms + k};
}

int ensure_tables(ixb_handle* h);

int ready(ixb_handle* h) {
  if (!h) return IXB_EINVAL;
  if (!h->has_mesh || !h->has_params || !h->has_bc[0] || !h->has_bc[1] || !h->has_bc[2]) return IXB_ESTATE;
  return ensure_tables(h);
}

// (Re)build the mesh-constant tables after a mesh or diffusivity change.
int ensure_tables(ixb_handle* h) {
  if (!h->tables_dirty) return IXB_OK;
  Geo<double> G = make_geo(h);
  CK(launch_tables_f64(G, h->metrics, h->tables, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->tables_dirty = false;
  return IXB_OK;
}


// Default launch shape of a sweep, from per-shape timings of every sweep on
// 64x64, 256x256 and 701x301 grids in both precision forms: x-lines one per
// CTA with 256 threads for lines of more than 384 rows, else 128; y-lines in
// the fused form with the fewest of 4, 5, 6 or 8 adjacent lines per CTA that
// keeps one CTA per SM (8 beyond that), and 128 threads per line for lines
// of 160 rows or more, else 64 (at 701x301: 5 x 128, one CTA on each of 141
// SMs, where 8 x 128 leaves 60 SMs idle; the u-y sweep measured 17.5 against
// 19.3 us, the other y-sweeps within 1 %).
// Those shapes were within about 5 % of the best (at worst 15 %, binary64
// y-sweeps at 701x301), where the rule below was 20-50 % behind.  When the
// shape cannot be resident: the fewest waves of CTAs, then the shortest
// chunks, then the most SMs busy (CTAs up to the SM count), then the larger CTA.
void pick_shape(ixb_handle* h, int eq) {
  {
    const bool x = (eq & 1) != 0;
    SweepShape probe = sweep_shape(eq, h->mi, h->nj, real_bytes(h), 1, 128);
    const int lines = probe.nfull, n = probe.n;
    int tl = 1;
    if (!x) {
      tl = 8;
      for (const int t : {4, 5, 6})
        if ((lines + t - 1) / t <= h->nsm) { tl = t; break; }
    }
    const int g = x ? (n > 384 ? 256 : 128) : (n >= 160 ? 128 : 64);
    const SweepShape s = sweep_shape(eq, h->mi, h->nj, real_bytes(h), tl, g);
    if (sweep_occupancy(eq, solver_form(h), s) > 0) {
      h->shape_tl[eq] = tl;
      h->shape_g[eq] = g;
      return;
    }
  }
  int best = -1;
  long long best_key = 0;
  for (int k = 0; k < kNumShapes; ++k) {
    SweepShape s = sweep_shape(eq, h->mi, h->nj, real_bytes(h), kShapeList[k][0], kShapeList[k][1]);
    const int occ = sweep_occupancy(eq, solver_form(h), s);
    if (occ <= 0) continue;
    const long long waves = (s.grid + (long long)occ * h->nsm - 1) / ((long long)occ * h->nsm);
    const long long busy = std::min<long long>(s.grid, h->nsm);
    const long long key = waves * 1000000000LL + (long long)s.m * 1000000 + (h->nsm - busy) * 1000 + (1024 - s.nt);
    if (best < 0 || key < best_key) { best = k; best_key = key; }
  }
  if (best < 0) best = 1;
  h->shape_tl[eq] = kShapeList[best][0];
  h->shape_g[eq] = kShapeList[best][1];
}

// Inputs and outputs of sweep `eq` at the handle's current buffer parity;
// flips the parity of the swept field (its output becomes current).
SweepIO<double> sweep_io(ixb_handle* h, int eq, const double* prev, bool with_norm) {
  SweepIO<double> io{};
  io.u = h->u[h->cu]; io.v = h->v[h->cv]; io.T = h->T[h->cT]; io.p = h->p; io.pc = h->pc[h->cpc];
  io.u_ant = h->u_ant; io.v_ant = h->v_ant; io.T_ant = h->T_ant;
  io.au = h->au; io.av = h->av;
  int var = -1;
  int* cur = nullptr;
  double** buf = nullptr;
  switch (eq) {
    case EQ_UY: case EQ_UX: var = 0; cur = &h->cu; buf = h->u; break;
    case EQ_VY: case EQ_VX: var = 1; cur = &h->cv; buf = h->v; break;
    case EQ_PY: case EQ_PX: var = -1; cur = &h->cpc; buf = h->pc; break;
    default: var = 2; cur = &h->cT; buf = h->T; break;
  }
  io.in = buf[*cur];
  io.out = buf[*cur ^ 1];
  io.prev = prev;
  io.fcon = io.flin = nullptr;  // an equation without sources reads none
  if (var >= 0) {
    if (h->fcon[var]) io.fcon = h->fcon[var];
    if (h->flin[var]) io.flin = h->flin[var];
    const bool x = (eq & 1) != 0;
    const BCEntry* base = h->bc + (size_t)var * 4 * h->bcstride;
    io.bc_first = base + (size_t)(x ? 0 : 1) * h->bcstride;
    io.bc_last = base + (size_t)(x ? 2 : 3) * h->bcstride;
  }
  if (eq == EQ_UX) io.aux = h->au;
  if (eq == EQ_VX) io.aux = h->av;
  if (eq == EQ_PX) io.aux = h->b_o;
  if (with_norm) {
    if (eq == EQ_VX) io.nrm0 = slot(h, N_DV);
    if (eq == EQ_PX) { io.nrm0 = slot(h, N_DP); io.nrm1 = slot(h, N_BO); }
    if (eq == EQ_TX) io.nrm0 = slot(h, N_DT);
  }
  *cur ^= 1;
  return io;
}

// Launch one sweep reading field buffers `cur` and writing `cur^1`; with
// zero_input the swept field is read as zeros (the handle's zero field),
// whatever its current buffer holds.
int sweep(ixb_handle* h, int eq, const double* prev, bool with_norm, const CtlRef& ctl = CtlRef{},
          bool zero_input = false, const ResidIO* rio = nullptr) {
  Geo<double> G = make_geo(h);
  if (h->shape_tl[eq] == 0) pick_shape(h, eq);
  SweepShape s = sweep_shape(eq, h->mi, h->nj, real_bytes(h), h->shape_tl[eq], h->shape_g[eq]);
  SweepIO<double> io = sweep_io(h, eq, prev, with_norm);
  if (zero_input) {
    io.in = h->zero;
    if (eq == EQ_PY || eq == EQ_PX) io.pc = h->zero;
  }
  const StageBuf stage{h->stage, h->stage_stride, h->stage_P};
  CK(launch_sweep_f64(eq, solver_form(h), s, G, io, stage, h->stream, ctl, rio));
  return IXB_OK;
}

// In the graph's do-while form the u residual and the outer test ride on
// every T-x sweep of the energy loop when that sweep runs fused: the
// residual of u-row jj reads T on row jj only, the line the sweep's CTA has
// just solved, so the separate residual kernel and its launch go away, and
// the last energy pass's values are the ones the outer test reads.
bool do_while_loops();
bool residual_in_tx(ixb_handle* h) {
  if (!h->use_graph || !do_while_loops()) return false;
  if (h->shape_tl[EQ_TX] == 0) pick_shape(h, EQ_TX);
  return fused_enabled() && fused_shape(EQ_TX, h->shape_tl[EQ_TX], h->shape_g[EQ_TX]);
}

int correct(ixb_handle* h, const CtlRef& gate = CtlRef{}) {
  Geo<double> G = make_geo(h);
  CK(launch_correct_f64(G, h->u[h->cu], h->v[h->cv], h->p, h->pc[h->cpc], h->au, h->av,
                         h->prm.solver == IXB_SOLVER_HYBRID, h->stream, gate));
  return IXB_OK;
}

int residual(ixb_handle* h, const CtlRef& outer = CtlRef{}) {
  Geo<double> G = make_geo(h);
  CK(launch_residual_f64(G, h->u[h->cu], h->v[h->cv], h->T[h->cT], h->p, h->u_ant, h->fcon[0], h->flin[0],
                         h->resu, slot(h, N_RES), h->prm.solver == IXB_SOLVER_HYBRID, h->stream, outer));
  return IXB_OK;
}

int read_norms(ixb_handle* h) {
  CK(cudaMemcpyAsync(h->h_norms, h->norms, N_COUNT * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return IXB_OK;
}

#define TRY(x)                 \
  do {                         \
    int s_ = (x);              \
    if (s_ != IXB_OK) return s_; \
  } while (0)

// ---------------------------------------------------------------------------
// host-driven body (one sync per inner pass), main.f90:404-1215
// ---------------------------------------------------------------------------
int body_host(ixb_handle* h, bool outer_test, ixb_report* rep, int* exit_code) {
  const ixb_params& P = h->prm;
  // ecuacion_momento
  for (;;) {
    TRY(sweep(h, EQ_UY, nullptr, false));
    TRY(sweep(h, EQ_UX, nullptr, false));
    const double* v_start = h->v[h->cv];
    TRY(sweep(h, EQ_VY, nullptr, false));
    TRY(sweep(h, EQ_VX, v_start, true));
    TRY(read_norms(h));
    const double err = h->h_norms[N_DV];
    rep->err_u = err;
    rep->n_momen++;
    if (!std::isfinite(err)) return IXB_ENONFINITE;
    if (err < P.conv_u) { h->iter_ecuaci = 0; break; }
    else if (h->iter_ecuaci > P.iter_ecuaci_max) { h->iter_ecuaci = 0; break; }
    else h->iter_ecuaci++;
  }
  // correccion_presion
  CK(cudaMemsetAsync(h->pc[h->cpc], 0, h->fsz * sizeof(double), h->stream));
  for (;;) {
    const double* pc_start = h->pc[h->cpc];
    TRY(sweep(h, EQ_PY, nullptr, false));
    TRY(sweep(h, EQ_PX, pc_start, true));
    TRY(read_norms(h));
    const double err = h->h_norms[N_DP];
    rep->err_p = err;
    rep->maxbo = h->h_norms[N_BO];
    rep->n_pres++;
    if (!std::isfinite(err) || !std::isfinite(rep->maxbo)) return IXB_ENONFINITE;
    if (err < P.conv_p) { h->iter_ecuaci = 0; break; }
    else if (h->iter_ecuaci > P.iter_ecuaci_max) { h->iter_ecuaci = 0; break; }
    else h->iter_ecuaci++;
  }
  TRY(correct(h));
  // solucion_energia
  for (;;) {
    const double* t_start = h->T[h->cT];
    TRY(sweep(h, EQ_TY, nullptr, false));
    TRY(sweep(h, EQ_TX, t_start, true));
    TRY(read_norms(h));
    const double err = h->h_norms[N_DT];
    rep->err_t = err;
    rep->n_ener++;
    if (!std::isfinite(err)) return IXB_ENONFINITE;
    if (err < P.conv_t) { h->iter_ecuaci = 0; break; }
    else if (h->iter_ecuaci > P.iter_ecuaci_max) { h->iter_ecuaci = 0; break; }
    else h->iter_ecuaci++;
  }
  TRY(residual(h));
  TRY(read_norms(h));
  rep->residuo = h->h_norms[N_RES];
  rep->n_simple++;
  if (!std::isfinite(rep->residuo)) return IXB_ENONFINITE;
  *exit_code = 0;
  if (!outer_test) return IXB_OK;
  if (rep->maxbo < P.conv_paso && rep->residuo < P.conv_resi) { h->iter_simple = 0; *exit_code = 1; }
  else if (h->iter_simple > P.iter_simple_max) { h->iter_simple = 0; *exit_code = 2; }
  else h->iter_simple++;
  return IXB_OK;
}

// ---------------------------------------------------------------------------
// graph-driven loop: control kernels set the WHILE conditions
// ---------------------------------------------------------------------------
__global__ void ctl_begin_kernel(Ctl* c, cudaGraphConditionalHandle outer) {
  IXB_PDL_ENTRY();
  cudaGraphSetConditional(outer, 1u);
  c->outer_done = 0;
  c->inner_done = 0;
  c->exit_code = 0;
  c->status = 0;
  c->n_simple = c->n_momen = c->n_pres = c->n_ener = 0;
}

// Counter of a K-pass WHILE loop: closes the loop after the pass that
// brings `left` to zero.
__global__ void loop_count_kernel(int* left, cudaGraphConditionalHandle cond) {
  if (--*left <= 0) cudaGraphSetConditional(cond, 0u);
}

// Add a WHILE node to `g` after `dep` and return its body graph.
int add_while(ixb_handle* h, cudaGraph_t g, cudaGraphNode_t* dep, cudaGraphConditionalHandle cond,
              cudaGraph_t* body, cudaGraphNode_t* node) {
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = cond;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  CK(cudaGraphAddNode(node, g, dep, dep ? 1 : 0, &np));
  *body = np.conditional.phGraph_out[0];
  return IXB_OK;
}

// Capture the launches issued by `fn` on the handle's stream into `g`,
// appended after the `ndep` nodes `deps` (or as roots); returns the last
// captured node (the capture's tail: `fn` issues its launches in order on
// one stream).
template <class F>
int capture_into_deps(ixb_handle* h, cudaGraph_t g, const cudaGraphNode_t* deps, size_t ndep, F fn,
                      cudaGraphNode_t* last, const cudaGraphEdgeData* edges = nullptr) {
  CK(cudaStreamBeginCaptureToGraph(h->stream, g, deps, edges, ndep, cudaStreamCaptureModeThreadLocal));
  int st = fn();
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const cudaGraphNode_t* tail = nullptr;
  size_t ntail = 0;
  cudaError_t ei = st == IXB_OK ? cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, nullptr, &tail, &ntail)
                                : cudaSuccess;
  *last = (ei == cudaSuccess && ntail == 1) ? tail[0] : nullptr;
  cudaGraph_t out = nullptr;
  cudaError_t e = cudaStreamEndCapture(h->stream, &out);
  if (st != IXB_OK) return st;
  CK(ei);
  CK(e);
  if (!*last) return IXB_ECUDA;  // nothing captured, or no single tail
  return IXB_OK;
}
template <class F>
int capture_into(ixb_handle* h, cudaGraph_t g, cudaGraphNode_t* dep, F fn, cudaGraphNode_t* last) {
  return capture_into_deps(h, g, dep, dep ? 1 : 0, fn, last);
}

// Inner loops in do-while form (the default): the first pass sits in the
// outer body, so the WHILE node launches its body only for further passes.
// With one pass per loop that took an outer iteration at 701x301 from 147
// to 136 us (refined) and from 156 to 150 us (binary64).  IXB_DOWHILE=0
// keeps every pass inside the WHILE node.
bool do_while_loops() {
  static const bool v = [] {
    const char* e = std::getenv("IXB_DOWHILE");
    return !(e && e[0] == '0');
  }();
  return v;
}

// Add the SIMPLE outer loop to graph `g` after `dep`: a WHILE node on
// `c_outer` (a conditional handle of `g`) whose body runs `unroll` outer
// passes.  unroll > 1 serves fixed counts that are multiples of it (every
// pass's outer test counts; the last one of the body decides whether it
// repeats).  Buffer parity must be 0 on entry (the passes return it to 0).
int add_outer_loop(ixb_handle* h, cudaGraph_t g, cudaGraphNode_t* dep, cudaGraphConditionalHandle c_outer,
                   int unroll, cudaGraphNode_t* n_outer) {
  // a conditional handle belongs to the graph that holds its node: the
  // outer handle to g, the inner ones to the outer loop's body
  cudaGraph_t outer_body;
  TRY(add_while(h, g, dep, c_outer, &outer_body, n_outer));
  cudaGraphNode_t last = nullptr, wn;
  cudaGraph_t b;
  const double* nrm = h->norms;
  for (int pass_no = 0; pass_no < unroll; ++pass_no) {
    cudaGraphConditionalHandle c_mom, c_pres, c_ener;
    CK(cudaGraphConditionalHandleCreate(&c_mom, outer_body, 1, cudaGraphCondAssignDefault));
    CK(cudaGraphConditionalHandleCreate(&c_pres, outer_body, 1, 0));
    CK(cudaGraphConditionalHandleCreate(&c_ener, outer_body, 1, 0));
    // outer pass: momentum loop -> pressure loop -> correct + gate(ener) -> energy loop
    //             -> residual + outer test.  Do-while form (the default): each loop is its
    //             first pass, then a WHILE node for further passes; the pressure loop's first
    //             pass reads p' as zero.  Otherwise: WHILE(mom) -> p' reset + gate(pres) ->
    //             WHILE(pres) -> ... with the momentum loop opened by the outer test of the
    //             previous pass and, for the first pass, by the handle's default.  The kernel
    //             that finishes a loop's norm applies its exit test (ixb_ctl.cuh).
    const auto mom_pass = [&]() -> int {
      TRY(sweep(h, EQ_UY, nullptr, false));
      TRY(sweep(h, EQ_UX, nullptr, false));
      const double* v_start = h->v[h->cv];
      TRY(sweep(h, EQ_VY, nullptr, false));
      TRY(sweep(h, EQ_VX, v_start, true, CtlRef{h->ctl_d, nrm, c_mom, 0, 0}));
      return IXB_OK;
    };
    const auto pres_pass = [&]() -> int {
      const double* pc_start = h->pc[h->cpc];
      TRY(sweep(h, EQ_PY, nullptr, false));
      TRY(sweep(h, EQ_PX, pc_start, true, CtlRef{h->ctl_d, nrm, c_pres, 0, 1}));
      return IXB_OK;
    };
    const bool res_tx = residual_in_tx(h);
    const ResidIO rio{h->u[h->cu], h->v[h->cv], h->p, h->u_ant, h->fcon[0], h->flin[0], h->resu, slot(h, N_RES),
                      CtlRef{h->ctl_d, nrm, c_outer, c_mom, 0}};
    const auto ener_pass = [&]() -> int {
      const double* t_start = h->T[h->cT];
      TRY(sweep(h, EQ_TY, nullptr, false));
      TRY(sweep(h, EQ_TX, t_start, true, CtlRef{h->ctl_d, nrm, c_ener, 0, 2}, false, res_tx ? &rio : nullptr));
      return IXB_OK;
    };
    const bool dw = do_while_loops();
    // one inner loop: WHILE(pass), or (do-while form) the first pass in the
    // outer body and a WHILE node for the further passes, whose condition the
    // first pass's exit test sets
    const auto inner_loop = [&](cudaGraphNode_t* dep, cudaGraphConditionalHandle cond, const auto& pass) -> int {
      if (dw) {
        TRY(capture_into(h, outer_body, dep, pass, &last));
        TRY(add_while(h, outer_body, &last, cond, &b, &wn));
      } else {
        TRY(add_while(h, outer_body, dep, cond, &b, &wn));
      }
      return capture_into(h, b, nullptr, pass, &last);
    };
    TRY(inner_loop(pass_no == 0 ? nullptr : &last, c_mom, mom_pass));
    if (dw) {
      // p' starts every pressure loop from zero (main.f90:752-758): the first
      // pass's y-sweep reads the zero field and its norm compares with zero,
      // so no reset kernel is needed; its exit test opens the WHILE node
      TRY(capture_into(h, outer_body, &wn, [&]() -> int {
        TRY(sweep(h, EQ_PY, nullptr, false, CtlRef{}, true));
        TRY(sweep(h, EQ_PX, h->zero, true, CtlRef{h->ctl_d, nrm, c_pres, 0, 1}));
        return IXB_OK;
      }, &last));
      TRY(add_while(h, outer_body, &last, c_pres, &b, &wn));
      TRY(capture_into(h, b, nullptr, pres_pass, &last));
    } else {
      TRY(capture_into(h, outer_body, &wn, [&]() {
        return launch_preset_f64(h->pc[h->cpc], h->fsz, CtlRef{h->ctl_d, nrm, c_pres, 0, 0}, h->stream) == cudaSuccess
                   ? IXB_OK : IXB_ECUDA;
      }, &last));
      TRY(inner_loop(&last, c_pres, pres_pass));
    }
    TRY(capture_into(h, outer_body, &wn, [&]() { return correct(h, CtlRef{h->ctl_d, nrm, c_ener, 0, 0}); }, &last));
    TRY(inner_loop(&last, c_ener, ener_pass));
    if (!res_tx)
      TRY(capture_into(h, outer_body, &wn, [&]() { return residual(h, CtlRef{h->ctl_d, nrm, c_outer, c_mom, 0}); },
                       &wn));
    last = wn;
  }
  return IXB_OK;
}

// Start of a block of outer passes inside the Nusselt monitor's loop: the
// block counts its passes from zero (fixed_count = the monitor's interval).
__global__ void block_begin_kernel(Ctl* c, cudaGraphConditionalHandle outer) {
  cudaGraphSetConditional(outer, 1u);
  c->outer_done = 0;
  c->inner_done = 0;
}

// The SIMPLE loop graphs.  GRAPH_PLAIN / GRAPH_UNROLLED: begin kernel, then
// the outer loop (1 or kOuterUnroll passes per WHILE body).  GRAPH_MON_*:
// begin kernel, then a WHILE node (the Nusselt monitor's loop) whose body is
// a block of outer passes (fixed_count of them, the monitor's interval) and
// the Nusselt kernel, whose monitor test decides whether another block runs.
int build_graph(ixb_handle* h, int kind, cudaGraph_t* graph, cudaGraphExec_t* exec) {
  if (*exec) { cudaGraphExecDestroy(*exec); *exec = nullptr; }
  if (*graph) { cudaGraphDestroy(*graph); *graph = nullptr; }
  const int unroll = (kind == GRAPH_UNROLLED || kind == GRAPH_MON_UNROLLED) ? kOuterUnroll : 1;
  const bool monitor = kind == GRAPH_MON_PLAIN || kind == GRAPH_MON_UNROLLED;
  // the graph bakes buffer parity 0 into its kernel arguments
  const int cu = h->cu, cv = h->cv, cT = h->cT, cpc = h->cpc;
  h->cu = h->cv = h->cT = h->cpc = 0;
  cudaGraph_t g;
  CK(cudaGraphCreate(&g, 0));
  *graph = g;
  cudaGraphConditionalHandle c_top;
  CK(cudaGraphConditionalHandleCreate(&c_top, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNode_t n_begin, n_top;
  TRY(capture_into(h, g, nullptr, [&]() {
    return launch_k(ctl_begin_kernel, 1, 1, 0, h->stream, h->ctl_d, c_top) == cudaSuccess ? IXB_OK : IXB_ECUDA;
  }, &n_begin));
  if (!monitor) {
    TRY(add_outer_loop(h, g, &n_begin, c_top, unroll, &n_top));
  } else {
    cudaGraph_t mbody;
    TRY(add_while(h, g, &n_begin, c_top, &mbody, &n_top));
    cudaGraphConditionalHandle c_outer;
    CK(cudaGraphConditionalHandleCreate(&c_outer, mbody, 1, cudaGraphCondAssignDefault));
    cudaGraphNode_t n_bb, n_outer, n_nu;
    TRY(capture_into(h, mbody, nullptr, [&]() {
      return launch_k(block_begin_kernel, 1, 1, 0, h->stream, h->ctl_d, c_outer) == cudaSuccess ? IXB_OK : IXB_ECUDA;
    }, &n_bb));
    TRY(add_outer_loop(h, mbody, &n_bb, c_outer, unroll, &n_outer));
    const Geo<double> G = make_geo(h);
    TRY(capture_into(h, mbody, &n_outer, [&]() {
      return launch_nusselt_f64(G, h->T[h->cT], h->xp_d, h->yp_d, 0, 1, 1, h->nu_d, h->stream, h->ctl_d, c_top) ==
                     cudaSuccess ? IXB_OK : IXB_ECUDA;
    }, &n_nu));
  }
  CK(cudaGraphInstantiate(exec, g, 0));
  h->cu = cu; h->cv = cv; h->cT = cT; h->cpc = cpc;
  return IXB_OK;
}

// The graph of `kind`, built or rebuilt when stale.
int ensure_graph(ixb_handle* h, int kind, cudaGraphExec_t* exec) {
  if (h->graph_dirty) {
    for (bool& st : h->graph_stale) st = true;
    h->graph_dirty = false;
  }
  cudaGraph_t* g = &h->graphs[kind];
  cudaGraphExec_t* e = &h->graph_execs[kind];
  if (h->graph_stale[kind] || !*e) {
    TRY(build_graph(h, kind, g, e));
    h->graph_stale[kind] = false;
  }
  *exec = *e;
  return IXB_OK;
}

// Bring every ping-pong field to buffer 0 (the parity the graph expects).
int normalize_parity(ixb_handle* h) {
  const size_t bytes = h->fsz * sizeof(double);
  if (h->cu) { CK(cudaMemcpyAsync(h->u[0], h->u[1], bytes, cudaMemcpyDeviceToDevice, h->stream)); h->cu = 0; }
  if (h->cv) { CK(cudaMemcpyAsync(h->v[0], h->v[1], bytes, cudaMemcpyDeviceToDevice, h->stream)); h->cv = 0; }
  if (h->cT) { CK(cudaMemcpyAsync(h->T[0], h->T[1], bytes, cudaMemcpyDeviceToDevice, h->stream)); h->cT = 0; }
  if (h->cpc) { CK(cudaMemcpyAsync(h->pc[0], h->pc[1], bytes, cudaMemcpyDeviceToDevice, h->stream)); h->cpc = 0; }
  return IXB_OK;
}

// Launch the graph of `kind` with the loop inputs of the handle; `mon`
// (monitor graphs only) sets the Nusselt monitor's inputs.
int run_graph_once(ixb_handle* h, int kind, int fixed_count, ixb_report* rep, const ixb_nu_monitor* mon = nullptr) {
  cudaGraphExec_t exec = nullptr;
  TRY(ensure_graph(h, kind, &exec));
  TRY(normalize_parity(h));
  Ctl* c = h->ctl_h;
  std::memset(c, 0, sizeof(Ctl));
  if (mon) {
    c->mon_vertical = mon->vertical;
    c->mon_k0 = mon->k0;
    c->mon_k1 = mon->k1;
    c->mon_wall = mon->wall;
    c->mon_max_iters = mon->max_iters;
    c->mon_tol_dnu = mon->tol_dnu;
    c->mon_tol_maxbo = mon->tol_maxbo;
  }
  c->conv_u = h->prm.conv_u; c->conv_p = h->prm.conv_p; c->conv_t = h->prm.conv_t;
  c->conv_resi = h->prm.conv_resi; c->conv_paso = h->prm.conv_paso;
  c->iter_ecuaci_max = h->prm.iter_ecuaci_max; c->iter_simple_max = h->prm.iter_simple_max;
  c->fixed_count = fixed_count;
  c->iter_ecuaci = h->iter_ecuaci;
  c->iter_simple = h->iter_simple;
  CK(cudaMemcpyAsync(h->ctl_d, c, sizeof(Ctl), cudaMemcpyHostToDevice, h->stream));
  CK(cudaGraphLaunch(exec, h->stream));
  CK(cudaMemcpyAsync(c, h->ctl_d, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  rep->maxbo = c->maxbo; rep->residuo = c->residuo;
  rep->err_u = c->err_u; rep->err_p = c->err_p; rep->err_t = c->err_t;
  rep->n_simple = c->n_simple; rep->n_momen = c->n_momen; rep->n_pres = c->n_pres; rep->n_ener = c->n_ener;
  rep->exit_code = c->exit_code;
  h->iter_ecuaci = c->iter_ecuaci;
  h->iter_simple = c->iter_simple;
  return c->status;
}

// The SIMPLE loop on the device: a fixed count that is a positive multiple
// of kOuterUnroll runs through the unrolled graph (one WHILE body launch per
// kOuterUnroll passes), anything else through the plain one.  (Splitting
// other counts into the two graphs costs a second launch and host sync per
// call, more than the unrolling saves on small grids.)
int run_graph(ixb_handle* h, int fixed_count, ixb_report* rep) {
  const bool unrolled = fixed_count > 0 && fixed_count % kOuterUnroll == 0;
  return run_graph_once(h, unrolled ? GRAPH_UNROLLED : GRAPH_PLAIN, fixed_count, rep);
}

void free_all(ixb_handle* h) {
  for (int k = 0; k < 4; ++k) {
    if (h->graph_execs[k]) cudaGraphExecDestroy(h->graph_execs[k]);
    if (h->graphs[k]) cudaGraphDestroy(h->graphs[k]);
  }
  if (h->egraph_exec) cudaGraphExecDestroy(h->egraph_exec);
  if (h->egraph) cudaGraphDestroy(h->egraph);
  if (h->agraph_exec) cudaGraphExecDestroy(h->agraph_exec);
  if (h->agraph) cudaGraphDestroy(h->agraph);
  if (h->loop_left) cudaFree(h->loop_left);
  double** bufs[] = {&h->u[0], &h->u[1], &h->v[0], &h->v[1], &h->T[0], &h->T[1], &h->pc[0], &h->pc[1],
                     &h->p, &h->u_ant, &h->v_ant, &h->T_ant, &h->au, &h->av, &h->b_o, &h->resu, &h->zero,
                     &h->fcon[0], &h->fcon[1], &h->fcon[2], &h->flin[0], &h->flin[1], &h->flin[2],
                     &h->metrics, &h->tables, &h->xp_d, &h->yp_d, &h->partials, &h->norms, &h->nu_d};
  for (auto b : bufs) if (*b) cudaFree(*b);
  if (h->stage) cudaFree(h->stage);
  if (h->adj_pool) cudaFree(h->adj_pool);
  if (h->xfer) cudaFree(h->xfer);
  if (h->dl_stream) cudaStreamSynchronize(h->dl_stream);
  if (h->snap) cudaFree(h->snap);
  if (h->snap_ev) cudaEventDestroy(h->snap_ev);
  if (h->dl_ev) cudaEventDestroy(h->dl_ev);
  if (h->dl_stream) cudaStreamDestroy(h->dl_stream);
  if (h->bc) cudaFree(h->bc);
  if (h->counters) cudaFree(h->counters);
  if (h->ctl_d) cudaFree(h->ctl_d);
  if (h->h_norms) cudaFreeHost(h->h_norms);
  if (h->ctl_h) cudaFreeHost(h->ctl_h);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
}

// The seven state arrays cross the bus as contiguous copies of their host
// (column-major, unpadded) layout through h->xfer, and one kernel moves all
// of them between that layout and the padded fields (pitched copies of
// ~5 KB rows ran at about 30 GB/s host->device).
struct XferSet {
  double* pad[7];    // padded device fields
  int rows[7], cols[7];
  size_t off[7];     // offset of array k in h->xfer
  int n;
};

__global__ void xfer_kernel(XferSet s, double* xfer, int LD, int to_padded) {
  const int k = blockIdx.y;
  const size_t total = (size_t)s.rows[k] * s.cols[k];
  double* flat = xfer + s.off[k];
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const size_t j = e / s.rows[k], i = e - j * s.rows[k];
    double* d = s.pad[k] + j * LD + i;
    if (to_padded) *d = flat[e];
    else flat[e] = *d;
  }
}

// The transfer set of the state arrays whose host pointer is not NULL, in
// the order u, v, p, T, u_ant, v_ant, T_ant, packed one after the other.
XferSet make_xfer_set(const ixb_handle* h, const std::array<double*, 7>& pad, const std::array<double*, 7>& host) {
  const int mi = h->mi, nj = h->nj;
  const int rows[7] = {mi, mi + 1, mi + 1, mi + 1, mi, mi + 1, mi + 1};
  const int cols[7] = {nj + 1, nj, nj + 1, nj + 1, nj + 1, nj, nj + 1};
  XferSet s{};
  size_t off = 0;
  for (int k = 0; k < 7; ++k) {
    if (!host[k]) continue;
    s.pad[s.n] = pad[k]; s.rows[s.n] = rows[k]; s.cols[s.n] = cols[k]; s.off[s.n] = off;
    off += (size_t)rows[k] * cols[k];
    ++s.n;
  }
  return s;
}

// host arrays (NULL: skipped) <-> the state fields
int xfer_state(ixb_handle* h, const std::array<double*, 7>& pad, const std::array<double*, 7>& host, bool upload) {
  const int mi = h->mi, nj = h->nj;
  const XferSet s = make_xfer_set(h, pad, host);
  if (s.n == 0) return IXB_OK;
  if (!h->xfer) {  // allocated on the first transfer (7 host-shaped arrays)
    CK(cudaStreamSynchronize(h->stream));
    if (cudaMalloc(&h->xfer, (size_t)7 * (mi + 1) * (nj + 1) * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      h->xfer = nullptr;
      return IXB_ENOMEM;
    }
  }
  const dim3 grid(148 * 2, s.n);
  if (upload) {
    for (int k = 0, q = 0; k < 7; ++k) {
      if (!host[k]) continue;
      CK(cudaMemcpyAsync(h->xfer + s.off[q], host[k], (size_t)s.rows[q] * s.cols[q] * sizeof(double),
                         cudaMemcpyHostToDevice, h->stream));
      ++q;
    }
    xfer_kernel<<<grid, 256, 0, h->stream>>>(s, h->xfer, h->LD, 1);
    CK(cudaGetLastError());
  } else {
    xfer_kernel<<<grid, 256, 0, h->stream>>>(s, h->xfer, h->LD, 0);
    CK(cudaGetLastError());
    for (int k = 0, q = 0; k < 7; ++k) {
      if (!host[k]) continue;
      CK(cudaMemcpyAsync(host[k], h->xfer + s.off[q], (size_t)s.rows[q] * s.cols[q] * sizeof(double),
                         cudaMemcpyDeviceToHost, h->stream));
      ++q;
    }
  }
  CK(cudaStreamSynchronize(h->stream));
  return IXB_OK;
}

// host Fortran array (rows x cols, column-major) <-> device padded field
int put2d(ixb_handle* h, double* dst, const double* src, int rows, int cols) {
  if (!src) return IXB_OK;
  CK(cudaMemcpy2DAsync(dst, (size_t)h->LD * sizeof(double), src, (size_t)rows * sizeof(double),
                       (size_t)rows * sizeof(double), cols, cudaMemcpyHostToDevice, h->stream));
  return IXB_OK;
}
int get2d(ixb_handle* h, double* dst, const double* src, int rows, int cols) {
  if (!dst) return IXB_OK;
  CK(cudaMemcpy2DAsync(dst, (size_t)rows * sizeof(double), src, (size_t)h->LD * sizeof(double),
                       (size_t)rows * sizeof(double), cols, cudaMemcpyDeviceToHost, h->stream));
  return IXB_OK;
}

// effective per-line boundary rows of one side: later segments overwrite
// earlier ones, as the sequential loop of impone_cond_frontera does
void side_table(const ixb_bc_side& s, BCEntry* tab, int nlines) {
  for (int L = 0; L < nlines; ++L) tab[L] = BCEntry{0.0, 0, 0};
  for (int k = 0; k < s.ndivis && k < 15; ++k) {
    const int t = s.type[k];
    if (t != IXB_BC_DIRI && t != IXB_BC_NEUM) continue;
    for (int L = s.index[k]; L <= s.index[k + 1]; ++L)
      if (L >= 1 && L < nlines) tab[L] = BCEntry{s.value[k], t, 0};
  }
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int ixb_version(void) { return 100; }

const char* ixb_strerror(int s) {
  switch (s) {
    case IXB_OK: return "ok";
    case IXB_EINVAL: return "invalid argument";
    case IXB_ECUDA: return "CUDA runtime error";
    case IXB_ENONFINITE: return "non-finite convergence norm";
    case IXB_ETIMEOUT: return "bounded device wait expired";
    case IXB_EBC: return "boundary table leaves a solved line without a boundary row";
    case IXB_ESTATE: return "mesh, parameters or boundary tables not set";
    case IXB_EIO: return "file read/parse/write error";
    case IXB_ENOMEM: return "allocation failed";
    default: return "unknown status";
  }
}

int ixb_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int ixb_create(int mi, int nj, int prec_mode, ixb_handle** out) {
  if (!out) return IXB_EINVAL;
  *out = nullptr;
  // a line of up to 6000 rows (chunks of <= 24 rows per thread) fits one CTA's shared memory
  if (mi < 4 || nj < 4 || mi > 6000 || nj > 6000) return IXB_EINVAL;
  if (prec_mode != IXB_PREC_FP64 && prec_mode != IXB_PREC_FP32_REFINED) return IXB_EINVAL;
  ixb_handle* h = new (std::nothrow) ixb_handle();
  if (!h) return IXB_ENOMEM;
  h->mi = mi; h->nj = nj; h->prec = prec_mode;
  h->LD = ((mi + 1) + 31) / 32 * 32;
  h->rows = nj + 2;
  h->fsz = (size_t)h->LD * h->rows;
  auto fail = [&](int code) { free_all(h); delete h; return code; };
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(IXB_ECUDA);
  h->own_stream = true;
  const size_t fb = h->fsz * sizeof(double);
  double** fields[] = {&h->u[0], &h->u[1], &h->v[0], &h->v[1], &h->T[0], &h->T[1], &h->pc[0], &h->pc[1],
                       &h->p, &h->u_ant, &h->v_ant, &h->T_ant, &h->au, &h->av, &h->b_o, &h->resu, &h->zero};
  for (auto f : fields) {
    if (cudaMalloc(f, fb) != cudaSuccess) return fail(IXB_ENOMEM);
    if (cudaMemset(*f, 0, fb) != cudaSuccess) return fail(IXB_ECUDA);
  }
  // au = av = 1e40 (main.f90:309-310)
  {
    std::vector<double> big(h->fsz, 1.e40);
    if (cudaMemcpy(h->au, big.data(), fb, cudaMemcpyHostToDevice) != cudaSuccess) return fail(IXB_ECUDA);
    if (cudaMemcpy(h->av, big.data(), fb, cudaMemcpyHostToDevice) != cudaSuccess) return fail(IXB_ECUDA);
  }
  h->mstride = std::max(mi, nj) + 3;
  if (cudaMalloc(&h->metrics, (size_t)M_COUNT * h->mstride * sizeof(double)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMemset(h->metrics, 0, (size_t)M_COUNT * h->mstride * sizeof(double)) != cudaSuccess) return fail(IXB_ECUDA);
  if (cudaMalloc(&h->tables, (size_t)T_COUNT * fb) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMemset(h->tables, 0, (size_t)T_COUNT * fb) != cudaSuccess) return fail(IXB_ECUDA);
  if (cudaMalloc(&h->xp_d, (size_t)h->mstride * sizeof(double)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMalloc(&h->yp_d, (size_t)h->mstride * sizeof(double)) != cudaSuccess) return fail(IXB_ENOMEM);
  h->bcstride = std::max(mi, nj) + 3;
  if (cudaMalloc(&h->bc, (size_t)12 * h->bcstride * sizeof(BCEntry)) != cudaSuccess) return fail(IXB_ENOMEM);
  cudaMemset(h->bc, 0, (size_t)12 * h->bcstride * sizeof(BCEntry));
  h->pstride = std::max(std::max(max_sweep_lines(mi, nj), residual_grid(mi, nj)), kAsmGridCap) + 32;
  // staged rows: up to max(mi, nj) + 2 lines of up to max(mi, nj) + 2 rows, binary64
  h->stage_P = (std::max(mi, nj) + 2 + 31) / 32 * 32;
  h->stage_stride = (size_t)max_sweep_lines(mi, nj) * h->stage_P;
  if (cudaMalloc(&h->stage, 4 * h->stage_stride * sizeof(double)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMalloc(&h->partials, (size_t)N_COUNT * h->pstride * sizeof(double)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMalloc(&h->counters, N_COUNT * sizeof(unsigned int)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMemset(h->counters, 0, N_COUNT * sizeof(unsigned int)) != cudaSuccess) return fail(IXB_ECUDA);
  if (cudaMalloc(&h->norms, N_COUNT * sizeof(double)) != cudaSuccess) return fail(IXB_ENOMEM);
  cudaMemset(h->norms, 0, N_COUNT * sizeof(double));
  if (cudaMalloc(&h->nu_d, 4 * sizeof(double)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMalloc(&h->ctl_d, sizeof(Ctl)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMallocHost(&h->h_norms, N_COUNT * sizeof(double)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMallocHost(&h->ctl_h, sizeof(Ctl)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (sweep_set_smem_limits() != cudaSuccess) return fail(IXB_ECUDA);
  {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return fail(IXB_ECUDA);
  }
  const char* env = std::getenv("IXB_NO_GRAPH");
  if (env && env[0] == '1') h->use_graph = 0;
  h->prm.p_update = 0.6;
  h->prm.solver = IXB_SOLVER_HYBRID;
  *out = h;
  return IXB_OK;
}

int ixb_destroy(ixb_handle* h) {
  if (!h) return IXB_EINVAL;
  if (h->stream) cudaStreamSynchronize(h->stream);
  free_all(h);
  delete h;
  return IXB_OK;
}

int ixb_set_stream(ixb_handle* h, void* stream) {
  if (!h) return IXB_EINVAL;
  CK(cudaStreamSynchronize(h->stream));
  if (h->own_stream) cudaStreamDestroy(h->stream);
  h->stream = (cudaStream_t)stream;
  h->own_stream = false;
  h->graph_dirty = h->egraph_dirty = h->agraph_dirty = true;
  return IXB_OK;
}

int ixb_set_mesh(ixb_handle* h, const double* xu, const double* yv, const double* xp, const double* yp) {
  if (!h || !xu || !yv || !xp || !yp) return IXB_EINVAL;
  const int mi = h->mi, nj = h->nj, ms = h->mstride;
  h->xu.assign(xu, xu + mi); h->yv.assign(yv, yv + nj);
  h->xp.assign(xp, xp + mi + 1); h->yp.assign(yp, yp + nj + 1);
  // 1-based views
  auto XU = [&](int i) { return xu[i - 1]; };
  auto YV = [&](int j) { return yv[j - 1]; };
  auto XP = [&](int i) { return xp[i - 1]; };
  auto YP = [&](int j) { return yp[j - 1]; };
  std::vector<double> m((size_t)M_COUNT * ms, 0.0);
  auto M = [&](int which, int k) -> double& { return m[(size_t)which * ms + k]; };
  // lectura_mallas_escalonadas, source/mod_malla.f90:167-218
  for (int ii = 2; ii <= mi; ++ii) M(M_DXP, ii) = XU(ii) - XU(ii - 1);
  for (int jj = 2; jj <= nj; ++jj) M(M_DYP, jj) = YV(jj) - YV(jj - 1);
  for (int ii = 1; ii <= mi; ++ii) M(M_DXU, ii) = XP(ii + 1) - XP(ii);
  for (int jj = 2; jj <= nj; ++jj) M(M_DYU, jj) = YV(jj) - YV(jj - 1);
  for (int ii = 2; ii <= mi; ++ii) M(M_DXV, ii) = XU(ii) - XU(ii - 1);
  for (int jj = 1; jj <= nj; ++jj) M(M_DYV, jj) = YP(jj + 1) - YP(jj);
  for (int ii = 1; ii <= mi; ++ii) M(M_FEXP, ii) = (XP(ii + 1) - XU(ii)) / (XP(ii + 1) - XP(ii));
  for (int jj = 1; jj <= nj; ++jj) M(M_FEYP, jj) = (YP(jj + 1) - YV(jj)) / (YP(jj + 1) - YP(jj));
  for (int ii = 1; ii <= mi - 1; ++ii) M(M_FEXU, ii) = (XU(ii + 1) - XP(ii + 1)) / (XU(ii + 1) - XU(ii));
  for (int jj = 1; jj <= nj - 1; ++jj) M(M_FEYV, jj) = (YV(jj + 1) - YP(jj + 1)) / (YV(jj + 1) - YV(jj));
  CK(cudaMemcpyAsync(h->metrics, m.data(), m.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  std::vector<double> xp1(ms, 0.0), yp1(ms, 0.0);
  for (int i = 1; i <= mi + 1; ++i) xp1[i] = XP(i);
  for (int j = 1; j <= nj + 1; ++j) yp1[j] = YP(j);
  CK(cudaMemcpyAsync(h->xp_d, xp1.data(), ms * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->yp_d, yp1.data(), ms * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->has_mesh = true;
  h->tables_dirty = true;
  return IXB_OK;
}

int ixb_set_params(ixb_handle* h, const ixb_params* p) {
  if (!h || !p) return IXB_EINVAL;
  if (p->solver != IXB_SOLVER_HYBRID && p->solver != IXB_SOLVER_EXACT) return IXB_EINVAL;
  if (!(p->dt != 0.0) || !(p->rel_vel != 0.0) || !(p->rel_pres != 0.0) || !(p->rel_ener != 0.0)) return IXB_EINVAL;
  if (p->gamma_momen != h->prm.gamma_momen || p->gamma_energ != h->prm.gamma_energ) h->tables_dirty = true;
  if (p->solver != h->prm.solver)
    for (int k = 0; k < EQ_COUNT; ++k) h->shape_tl[k] = h->shape_g[k] = 0;
  h->prm = *p;
  h->has_params = true;
  h->graph_dirty = h->egraph_dirty = h->agraph_dirty = true;
  return IXB_OK;
}

int ixb_set_bc(ixb_handle* h, int var, const ixb_bc_side sides[4]) {
  if (!h || !sides || var < 0 || var > 2) return IXB_EINVAL;
  const int mi = h->mi, nj = h->nj, S = h->bcstride;
  std::vector<BCEntry> tab((size_t)4 * S);
  for (int k = 0; k < 4; ++k) {
    const ixb_bc_side& s = sides[k];
    if (s.side < 0 || s.side > 3 || s.ndivis < 0 || s.ndivis > 15) return IXB_EINVAL;
  }
  for (int side = 0; side < 4; ++side) {
    // a side entry may appear anywhere in the array; the last one for a side wins
    const ixb_bc_side* s = nullptr;
    for (int k = 0; k < 4; ++k) if (sides[k].side == side) s = &sides[k];
    BCEntry* t = tab.data() + (size_t)side * S;
    if (s) side_table(*s, t, S);
    else for (int L = 0; L < S; ++L) t[L] = BCEntry{0.0, 0, 0};
    // solved lines of this side: x-lines (a, c) and y-lines (b, d) of the variable
    int lo = 2, hi;
    const bool xside = (side == 0 || side == 2);
    if (var == 0) hi = xside ? nj : mi - 1;       // u: x-lines jj=2..nj, y-lines ii=2..mi-1
    else if (var == 1) hi = xside ? nj - 1 : mi;  // v: jj=2..nj-1, ii=2..mi
    else hi = xside ? nj : mi;                    // T: jj=2..nj, ii=2..mi
    for (int L = lo; L <= hi; ++L)
      if (t[L].type != IXB_BC_DIRI && t[L].type != IXB_BC_NEUM) return IXB_EBC;
  }
  CK(cudaMemcpyAsync(h->bc + (size_t)var * 4 * S, tab.data(), tab.size() * sizeof(BCEntry),
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->has_bc[var] = true;
  return IXB_OK;
}

int ixb_set_sources(ixb_handle* h, int var, const double* fcon, const double* flin) {
  if (!h || var < 0 || var > 2) return IXB_EINVAL;
  const int rows = var == 0 ? h->mi : h->mi + 1;
  const int cols = var == 1 ? h->nj : h->nj + 1;
  const size_t fb = h->fsz * sizeof(double);
  double** pc[2] = {&h->fcon[var], &h->flin[var]};
  const double* src[2] = {fcon, flin};
  for (int k = 0; k < 2; ++k) {
    if (!src[k]) {
      if (*pc[k]) { cudaFree(*pc[k]); *pc[k] = nullptr; }
      continue;
    }
    if (!*pc[k]) {
      if (cudaMalloc(pc[k], fb) != cudaSuccess) return IXB_ENOMEM;
      CK(cudaMemset(*pc[k], 0, fb));
    }
    TRY(put2d(h, *pc[k], src[k], rows, cols));
  }
  CK(cudaStreamSynchronize(h->stream));
  h->graph_dirty = h->egraph_dirty = h->agraph_dirty = true;
  return IXB_OK;
}

int ixb_upload_state(ixb_handle* h, const double* u, const double* v, const double* p, const double* T,
                     const double* u_ant, const double* v_ant, const double* T_ant) {
  if (!h) return IXB_EINVAL;
  return xfer_state(h, {h->u[h->cu], h->v[h->cv], h->p, h->T[h->cT], h->u_ant, h->v_ant, h->T_ant},
                    {const_cast<double*>(u), const_cast<double*>(v), const_cast<double*>(p), const_cast<double*>(T),
                     const_cast<double*>(u_ant), const_cast<double*>(v_ant), const_cast<double*>(T_ant)},
                    true);
}

int ixb_download_state(ixb_handle* h, double* u, double* v, double* p, double* T, double* u_ant, double* v_ant,
                       double* T_ant) {
  if (!h) return IXB_EINVAL;
  return xfer_state(h, {h->u[h->cu], h->v[h->cv], h->p, h->T[h->cT], h->u_ant, h->v_ant, h->T_ant},
                    {u, v, p, T, u_ant, v_ant, T_ant}, false);
}

int ixb_download_state_async(ixb_handle* h, double* u, double* v, double* p, double* T, double* u_ant,
                             double* v_ant, double* T_ant) {
  if (!h) return IXB_EINVAL;
  const std::array<double*, 7> host = {u, v, p, T, u_ant, v_ant, T_ant};
  const XferSet s = make_xfer_set(h, {h->u[h->cu], h->v[h->cv], h->p, h->T[h->cT], h->u_ant, h->v_ant, h->T_ant},
                                  host);
  if (s.n == 0) return IXB_OK;
  if (!h->snap) {  // first use: the snapshot buffer, the download stream and its events
    CK(cudaStreamSynchronize(h->stream));
    if (cudaMalloc(&h->snap, (size_t)7 * (h->mi + 1) * (h->nj + 1) * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      h->snap = nullptr;
      return IXB_ENOMEM;
    }
    CK(cudaStreamCreateWithFlags(&h->dl_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h->snap_ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->dl_ev, cudaEventDisableTiming));
  }
  // the snapshot buffer is reused once the previous download has read it
  if (h->dl_pending) CK(cudaStreamWaitEvent(h->stream, h->dl_ev, 0));
  const dim3 grid(148 * 2, s.n);
  xfer_kernel<<<grid, 256, 0, h->stream>>>(s, h->snap, h->LD, 0);
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->snap_ev, h->stream));
  CK(cudaStreamWaitEvent(h->dl_stream, h->snap_ev, 0));
  for (int k = 0, q = 0; k < 7; ++k) {
    if (!host[k]) continue;
    CK(cudaMemcpyAsync(host[k], h->snap + s.off[q], (size_t)s.rows[q] * s.cols[q] * sizeof(double),
                       cudaMemcpyDeviceToHost, h->dl_stream));
    ++q;
  }
  CK(cudaEventRecord(h->dl_ev, h->dl_stream));
  h->dl_pending = true;
  return IXB_OK;
}

int ixb_download_wait(ixb_handle* h) {
  if (!h) return IXB_EINVAL;
  if (!h->dl_pending) return IXB_OK;
  CK(cudaEventSynchronize(h->dl_ev));
  return IXB_OK;
}

int ixb_host_alloc(size_t bytes, void** out) {
  if (!out || bytes == 0) return IXB_EINVAL;
  *out = nullptr;
  if (cudaMallocHost(out, bytes) != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return IXB_ENOMEM;
  }
  return IXB_OK;
}

int ixb_host_free(void* p) {
  if (p && cudaFreeHost(p) != cudaSuccess) return IXB_ECUDA;
  return IXB_OK;
}

int ixb_download_aux(ixb_handle* h, double* au, double* av, double* b_o, double* resu, double* corr_pres) {
  if (!h) return IXB_EINVAL;
  const int mi = h->mi, nj = h->nj;
  TRY(get2d(h, au, h->au, mi, nj + 1));
  TRY(get2d(h, av, h->av, mi + 1, nj));
  TRY(get2d(h, b_o, h->b_o, mi + 1, nj + 1));
  TRY(get2d(h, resu, h->resu, mi, nj + 1));
  TRY(get2d(h, corr_pres, h->pc[h->cpc], mi + 1, nj + 1));
  CK(cudaStreamSynchronize(h->stream));
  return IXB_OK;
}

int ixb_set_work(ixb_handle* h, const double* corr_pres, const double* au, const double* av) {
  if (!h) return IXB_EINVAL;
  const int mi = h->mi, nj = h->nj;
  TRY(put2d(h, h->pc[h->cpc], corr_pres, mi + 1, nj + 1));
  TRY(put2d(h, h->au, au, mi, nj + 1));
  TRY(put2d(h, h->av, av, mi + 1, nj));
  CK(cudaStreamSynchronize(h->stream));
  return IXB_OK;
}

static void rep_clear(ixb_report* r) { std::memset(r, 0, sizeof(*r)); }

int ixb_simple_iterations(ixb_handle* h, int n, ixb_report* rep) {
  TRY(ready(h));
  if (n < 0) return IXB_EINVAL;
  ixb_report local;
  ixb_report* r = rep ? rep : &local;
  rep_clear(r);
  if (n == 0) return IXB_OK;
  int st;
  if (h->use_graph) {
    st = run_graph(h, n, r);
  } else {
    st = IXB_OK;
    int code = 0;
    for (int k = 0; k < n && st == IXB_OK; ++k) st = body_host(h, false, r, &code);
    if (st == IXB_OK) CK(cudaStreamSynchronize(h->stream));
  }
  r->status = st;
  return st;
}

int ixb_simple_loop(ixb_handle* h, ixb_report* rep) {
  TRY(ready(h));
  ixb_report local;
  ixb_report* r = rep ? rep : &local;
  rep_clear(r);
  int st;
  if (h->use_graph) {
    st = run_graph(h, 0, r);
  } else {
    st = IXB_OK;
    int code = 0;
    while (st == IXB_OK) {
      st = body_host(h, true, r, &code);
      if (code != 0) break;
    }
    r->exit_code = code;
  }
  r->status = st;
  return st;
}

static int nusselt(ixb_handle* h, int vertical, int k0, int k1, double* nu0, double* nu1);

// Panels k0..k1 (step 2) of a wall-averaged Nusselt number fit the walls.
static bool nu_range_ok(const ixb_handle* h, int vertical, int k0, int k1) {
  const int n_along = vertical ? h->nj + 1 : h->mi + 1;
  if (k0 < 1 || k1 < k0) return false;
  return k0 + 2 * ((k1 - k0) / 2) + 2 <= n_along;
}

int ixb_simple_converge(ixb_handle* h, const ixb_nu_monitor* mon, ixb_report* rep, double* nu, double* dnu) {
  TRY(ready(h));
  if (!mon || mon->every < 1 || mon->max_iters < 1 || (mon->vertical != 0 && mon->vertical != 1) ||
      (mon->wall != 0 && mon->wall != 1) || !(mon->tol_dnu >= 0.0) || !(mon->tol_maxbo >= 0.0) ||
      !nu_range_ok(h, mon->vertical, mon->k0, mon->k1))
    return IXB_EINVAL;
  ixb_report local;
  ixb_report* r = rep ? rep : &local;
  rep_clear(r);
  double nu2[2] = {0.0, 0.0}, d = INFINITY;
  int st;
  if (h->use_graph) {
    const int kind = mon->every % kOuterUnroll == 0 ? GRAPH_MON_UNROLLED : GRAPH_MON_PLAIN;
    st = run_graph_once(h, kind, mon->every, r, mon);
    const Ctl* c = h->ctl_h;
    nu2[0] = c->mon_nu[0];
    nu2[1] = c->mon_nu[1];
    d = c->mon_dnu;
  } else {
    // host-driven: blocks of `every` passes, the Nusselt number and the
    // monitor's test on the host, in the order the graph applies them
    st = IXB_OK;
    long long evals = 0;
    double prev = 0.0;
    while (st == IXB_OK) {
      ixb_report b;
      st = ixb_simple_iterations(h, mon->every, &b);
      r->n_simple += b.n_simple; r->n_momen += b.n_momen; r->n_pres += b.n_pres; r->n_ener += b.n_ener;
      r->maxbo = b.maxbo; r->residuo = b.residuo; r->err_u = b.err_u; r->err_p = b.err_p; r->err_t = b.err_t;
      if (st != IXB_OK) break;
      st = nusselt(h, mon->vertical, mon->k0, mon->k1, &nu2[0], &nu2[1]);
      if (st != IXB_OK) break;
      const double v = nu2[mon->wall];
      d = evals > 0 ? std::fabs(v - prev) : INFINITY;
      prev = v;
      ++evals;
      if (!std::isfinite(v)) { st = IXB_ENONFINITE; break; }
      if (d < mon->tol_dnu) { r->exit_code = 3; break; }
      if (r->maxbo < mon->tol_maxbo) { r->exit_code = 4; break; }
      if (r->n_simple >= mon->max_iters) { r->exit_code = 5; break; }
    }
  }
  if (nu) { nu[0] = nu2[0]; nu[1] = nu2[1]; }
  if (dnu) *dnu = d;
  r->status = st;
  return st;
}

int ixb_roll(ixb_handle* h) {
  if (!h) return IXB_EINVAL;
  const size_t fb = h->fsz * sizeof(double);
  CK(cudaMemcpyAsync(h->T_ant, h->T[h->cT], fb, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(h->u_ant, h->u[h->cu], fb, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(h->v_ant, h->v[h->cv], fb, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return IXB_OK;
}

int ixb_step(ixb_handle* h, ixb_report* rep) {
  TRY(ixb_simple_loop(h, rep));
  return ixb_roll(h);
}

int ixb_phase(ixb_handle* h, int which) {
  TRY(ready(h));
  int st = IXB_OK;
  switch (which) {
    case 0: st = sweep(h, EQ_UY, nullptr, false); break;
    case 1: st = sweep(h, EQ_UX, nullptr, false); break;
    case 2: st = sweep(h, EQ_VY, nullptr, false); break;
    case 3: st = sweep(h, EQ_VX, nullptr, false); break;
    case 4: st = sweep(h, EQ_PY, nullptr, false); break;
    case 5: st = sweep(h, EQ_PX, nullptr, false); break;
    case 6: st = correct(h); break;
    case 7: st = sweep(h, EQ_TY, nullptr, false); break;
    case 8: st = sweep(h, EQ_TX, nullptr, false); break;
    case 9: st = residual(h); break;
    default: return IXB_EINVAL;
  }
  if (st != IXB_OK) return st;
  CK(cudaStreamSynchronize(h->stream));
  return IXB_OK;
}

int ixb_time_phases(ixb_handle* h, int reps, size_t flush_bytes, double* ms) {
  TRY(ready(h));
  if (reps < 1 || !ms) return IXB_EINVAL;
  void* flush = nullptr;
  if (flush_bytes > 0 && cudaMalloc(&flush, flush_bytes) != cudaSuccess) return IXB_ENOMEM;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int st = IXB_OK;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) st = IXB_ECUDA;
  for (int k = 0; k < 10 && st == IXB_OK; ++k) {
    auto launch = [&]() -> int {
      switch (k) {
        case 0: return sweep(h, EQ_UY, nullptr, false);
        case 1: return sweep(h, EQ_UX, nullptr, false);
        case 2: return sweep(h, EQ_VY, nullptr, false);
        case 3: return sweep(h, EQ_VX, h->v[h->cv ^ 1], true);
        case 4: return sweep(h, EQ_PY, nullptr, false);
        case 5: return sweep(h, EQ_PX, h->pc[h->cpc ^ 1], true);
        case 6: return correct(h);
        case 7: return sweep(h, EQ_TY, nullptr, false);
        case 8: return sweep(h, EQ_TX, h->T[h->cT ^ 1], true);
        default: return residual(h);
      }
    };
    st = launch();  // warm-up (module load, first-touch)
    double total = 0.0;
    for (int r = 0; r < reps && st == IXB_OK; ++r) {
      if (flush && cudaMemsetAsync(flush, r & 0xff, flush_bytes, h->stream) != cudaSuccess) { st = IXB_ECUDA; break; }
      if (cudaEventRecord(e0, h->stream) != cudaSuccess) { st = IXB_ECUDA; break; }
      st = launch();
      if (st != IXB_OK) break;
      if (cudaEventRecord(e1, h->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
        st = IXB_ECUDA;
        break;
      }
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      total += t;
    }
    ms[k] = total / reps;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (flush) cudaFree(flush);
  return st;
}

int ixb_iteration_launches(ixb_handle* h, int* launches) {
  if (!h || !launches) return IXB_EINVAL;
  // p/u/v correction, u residual, and the p' reset kernel unless the graph
  // runs the inner loops in do-while form (whose first pressure pass reads zeros)
  int k = (h->use_graph && do_while_loops()) ? 2 : 3;
  if (residual_in_tx(h)) k -= 1;  // the u residual rides on the fused T-x sweep
  for (int eq = 0; eq < EQ_COUNT; ++eq) {
    if (h->shape_tl[eq] == 0) pick_shape(h, eq);
    k += (fused_enabled() && fused_shape(eq, h->shape_tl[eq], h->shape_g[eq])) ? 1 : 2;
  }
  *launches = k;
  return IXB_OK;
}

int ixb_set_sweep_shape(ixb_handle* h, int sweep, int lines_per_cta, int threads_per_line) {
  if (!h || sweep < 0 || sweep >= EQ_COUNT) return IXB_EINVAL;
  if (lines_per_cta == 0) {  // back to the default choice
    h->shape_tl[sweep] = h->shape_g[sweep] = 0;
    h->graph_dirty = h->egraph_dirty = h->agraph_dirty = true;
    return IXB_OK;
  }
  int k = 0;
  for (; k < kNumShapes; ++k)
    if (kShapeList[k][0] == lines_per_cta && kShapeList[k][1] == threads_per_line) break;
  if (k == kNumShapes) return IXB_EINVAL;
  SweepShape s = sweep_shape(sweep, h->mi, h->nj, real_bytes(h), lines_per_cta, threads_per_line);
  if (sweep_occupancy(sweep, solver_form(h), s) <= 0) return IXB_EINVAL;
  h->shape_tl[sweep] = lines_per_cta;
  h->shape_g[sweep] = threads_per_line;
  h->graph_dirty = h->egraph_dirty = h->agraph_dirty = true;
  return IXB_OK;
}

int ixb_autotune(ixb_handle* h, int reps, size_t flush_bytes, int* chosen, double* ms) {
  TRY(ready(h));
  if (reps < 1) return IXB_EINVAL;
  // save the state the timing launches overwrite
  const size_t fb = h->fsz * sizeof(double);
  double* save = nullptr;
  const int nsave = 11;
  double* bufs[nsave] = {h->u[0], h->u[1], h->v[0], h->v[1], h->T[0], h->T[1], h->pc[0], h->pc[1],
                         h->au, h->av, h->b_o};
  if (cudaMalloc(&save, nsave * fb) != cudaSuccess) return IXB_ENOMEM;
  void* flush = nullptr;
  if (flush_bytes > 0 && cudaMalloc(&flush, flush_bytes) != cudaSuccess) { cudaFree(save); return IXB_ENOMEM; }
  const int cu = h->cu, cv = h->cv, cT = h->cT, cpc = h->cpc;
  int st = IXB_OK;
  for (int k = 0; k < nsave && st == IXB_OK; ++k)
    if (cudaMemcpyAsync(save + k * h->fsz, bufs[k], fb, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess)
      st = IXB_ECUDA;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (st == IXB_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) st = IXB_ECUDA;
  for (int eq = 0; eq < EQ_COUNT && st == IXB_OK; ++eq) {
    double best = 1e30;
    int best_k = -1;
    for (int k = 0; k < kNumShapes && st == IXB_OK; ++k) {
      if (ixb_set_sweep_shape(h, eq, kShapeList[k][0], kShapeList[k][1]) != IXB_OK) continue;
      st = sweep(h, eq, nullptr, false);  // warm-up
      double total = 0.0;
      for (int r = 0; r < reps && st == IXB_OK; ++r) {
        if (flush && cudaMemsetAsync(flush, r & 0xff, flush_bytes, h->stream) != cudaSuccess) { st = IXB_ECUDA; break; }
        if (cudaEventRecord(e0, h->stream) != cudaSuccess) { st = IXB_ECUDA; break; }
        st = sweep(h, eq, nullptr, false);
        if (st != IXB_OK) break;
        if (cudaEventRecord(e1, h->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
          st = IXB_ECUDA;
          break;
        }
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        total += t;
      }
      const double mean = total / reps;
      if (st == IXB_OK && mean < best) { best = mean; best_k = k; }
    }
    if (st != IXB_OK) break;
    if (best_k < 0) { st = IXB_ECUDA; break; }
    h->shape_tl[eq] = kShapeList[best_k][0];
    h->shape_g[eq] = kShapeList[best_k][1];
    if (chosen) { chosen[2 * eq] = kShapeList[best_k][0]; chosen[2 * eq + 1] = kShapeList[best_k][1]; }
    if (ms) ms[eq] = best;
  }
  for (int k = 0; k < nsave; ++k)
    cudaMemcpyAsync(bufs[k], save + k * h->fsz, fb, cudaMemcpyDeviceToDevice, h->stream);
  h->cu = cu; h->cv = cv; h->cT = cT; h->cpc = cpc;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess && st == IXB_OK) st = IXB_ECUDA;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (flush) cudaFree(flush);
  cudaFree(save);
  h->graph_dirty = h->egraph_dirty = h->agraph_dirty = true;
  return st;
}

static int nusselt(ixb_handle* h, int vertical, int k0, int k1, double* nu0, double* nu1) {
  if (!h || !h->has_mesh) return IXB_ESTATE;
  if (!nu_range_ok(h, vertical, k0, k1)) return IXB_EINVAL;
  Geo<double> G = make_geo(h);
  CK(launch_nusselt_f64(G, h->T[h->cT], h->xp_d, h->yp_d, vertical, k0, k1, h->nu_d, h->stream));
  double out[2];
  CK(cudaMemcpyAsync(out, h->nu_d, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (nu0) *nu0 = out[0];
  if (nu1) *nu1 = out[1];
  return IXB_OK;
}

int ixb_energy_iterations(ixb_handle* h, int n) {
  if (!h || n < 0) return IXB_EINVAL;
  TRY(ready(h));
  if (n == 0) return IXB_OK;
  // one pass, T-y then T-x (buffer parity back to 0); kLoopUnroll of them
  // form the body of a WHILE loop, the rest run as plain launches
  const std::function<int()> pass = [h]() -> int {
    TRY(sweep(h, EQ_TY, nullptr, false));
    return sweep(h, EQ_TX, nullptr, false);
  };
  if (h->egraph_dirty || !h->egraph_exec) {
    TRY(handle_build_loop_graph(h, pass, kLoopUnroll, &h->egraph, &h->egraph_exec));
    h->egraph_dirty = false;
  }
  if (n >= kLoopUnroll) TRY(handle_run_loop_graph(h, h->egraph_exec, n / kLoopUnroll));
  for (int k = 0; k < n % kLoopUnroll; ++k) TRY(pass());
  CK(cudaStreamSynchronize(h->stream));
  return IXB_OK;
}

int ixb_set_bc_values(ixb_handle* h, int var, int side, const double* values) {
  if (!h || !values || var < 0 || var > 2 || side < 0 || side > 3) return IXB_EINVAL;
  if (!h->has_bc[var]) return IXB_ESTATE;
  const int nl = (side == 0 || side == 2) ? (var == 1 ? h->nj : h->nj + 1) : (var == 0 ? h->mi : h->mi + 1);
  std::vector<BCEntry> e(nl + 1);
  BCEntry* d = h->bc + ((size_t)var * 4 + side) * h->bcstride;
  CK(cudaMemcpyAsync(e.data(), d, e.size() * sizeof(BCEntry), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int l = 1; l <= nl; ++l) e[l].val = values[l - 1];
  CK(cudaMemcpyAsync(d, e.data(), e.size() * sizeof(BCEntry), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return IXB_OK;
}

int ixb_nusselt_y(ixb_handle* h, int i0, int i1, double* nu0, double* nu1) { return nusselt(h, 0, i0, i1, nu0, nu1); }
int ixb_nusselt_x(ixb_handle* h, int j0, int j1, double* nu0, double* nu1) { return nusselt(h, 1, j0, j1, nu0, nu1); }

int ixb_tridiag_f64(const double* a, const double* b, const double* c, const double* d, double* x, int n, int nsys,
                    int layout, int solver, void* stream) {
  if (!a || !b || !c || !d || !x || n < 1 || nsys < 1 || (layout != 0 && layout != 1)) return IXB_EINVAL;
  if (solver != IXB_SOLVER_HYBRID && solver != IXB_SOLVER_EXACT) return IXB_EINVAL;
  cudaError_t e = tridiag_f64(a, b, c, d, x, n, nsys, layout, solver, (cudaStream_t)stream);
  if (e == cudaErrorInvalidValue) return IXB_EINVAL;
  return e == cudaSuccess ? IXB_OK : IXB_ECUDA;
}

int ixb_tridiag_f32(const float* a, const float* b, const float* c, const float* d, float* x, int n, int nsys,
                    int layout, int solver, void* stream) {
  if (!a || !b || !c || !d || !x || n < 1 || nsys < 1 || (layout != 0 && layout != 1)) return IXB_EINVAL;
  if (solver != IXB_SOLVER_HYBRID && solver != IXB_SOLVER_EXACT) return IXB_EINVAL;
  cudaError_t e = tridiag_f32(a, b, c, d, x, n, nsys, layout, solver, (cudaStream_t)stream);
  if (e == cudaErrorInvalidValue) return IXB_EINVAL;
  return e == cudaSuccess ? IXB_OK : IXB_ECUDA;
}

int ixb_tridiag_status(void) {
  if (cudaDeviceSynchronize() != cudaSuccess) return IXB_ECUDA;
  int flag = 0;
  if (tridiag_take_timeout(&flag) != cudaSuccess) return IXB_ECUDA;
  return flag ? IXB_ETIMEOUT : IXB_OK;
}

}  // extern "C"

namespace ixb {
int handle_build_loop_graph(ixb_handle* h, const std::function<int()>& pass, int unroll, cudaGraph_t* graph,
                            cudaGraphExec_t* exec) {
  if (*exec) { cudaGraphExecDestroy(*exec); *exec = nullptr; }
  if (*graph) { cudaGraphDestroy(*graph); *graph = nullptr; }
  if (!h->loop_left && cudaMalloc(&h->loop_left, sizeof(int)) != cudaSuccess) return IXB_ENOMEM;
  TRY(normalize_parity(h));
  cudaGraph_t g;
  CK(cudaGraphCreate(&g, 0));
  *graph = g;
  cudaGraphConditionalHandle c;
  CK(cudaGraphConditionalHandleCreate(&c, g, 1, cudaGraphCondAssignDefault));
  cudaGraph_t body;
  cudaGraphNode_t wnode, last;
  TRY(add_while(h, g, nullptr, c, &body, &wnode));
  TRY(capture_into(h, body, nullptr, [&]() -> int {
    for (int u = 0; u < unroll; ++u) TRY(pass());
    loop_count_kernel<<<1, 1, 0, h->stream>>>(h->loop_left, c);
    return cudaGetLastError() == cudaSuccess ? IXB_OK : IXB_ECUDA;
  }, &last));
  CK(cudaGraphInstantiate(exec, g, 0));
  return IXB_OK;
}
int handle_run_loop_graph(ixb_handle* h, cudaGraphExec_t exec, int passes) {
  TRY(normalize_parity(h));
  CK(cudaMemcpyAsync(h->loop_left, &passes, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  CK(cudaGraphLaunch(exec, h->stream));
  return IXB_OK;
}
Geo<double> handle_geo(const ixb_handle* h) { return make_geo(h); }
int handle_solver_form(const ixb_handle* h) { return solver_form(h); }
int handle_ready(ixb_handle* h) { return ready(h); }
SweepIO<double> handle_sweep_io(ixb_handle* h, int eq, const double* prev) { return sweep_io(h, eq, prev, false); }
int handle_real_bytes(const ixb_handle* h) { return real_bytes(h); }
}  // namespace ixb
