// ixb_batch.cu -- many SIMPLE instances (cavities of different sizes and
// parameters) advanced together: every phase of the outer iteration is one
// launch over the work items of all instances (assembly tiles, line groups,
// cell blocks), and the whole loop is one CUDA graph with a WHILE node whose
// condition a control kernel sets on the device.
//
// The reference runs one case per process (PROGRAM IXCHEL2D, source/main.f90);
// this driver has no counterpart there.  Each instance is an ordinary
// ixb_handle (its buffers, mesh tables, boundary tables and state are set up
// through the single-instance calls); the batch only adds the batched
// launches.  An outer iteration here is one pass of each equation (the
// reference's loops with iter_ecuaci_max = 0); an instance stops when its
// outer test of main.f90:1202 holds (maxbo < conv_paso and residuo <
// conv_resi), on a non-finite norm, or when the call's iteration budget is
// spent.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <type_traits>
#include <vector>

#include "ixb_handle.h"
#include "ixb_reduce.cuh"

using namespace ixb;

namespace {

// per-instance loop state on the device
struct BInst {
  int iters;       // outer iterations done since the last restart
  int exit_code;   // 0 running, 1 outer test met, 2 stopped by the iteration budget, 3 non-finite norm
  int status;      // IXB_OK or IXB_ENONFINITE
  int pad;
  double conv_paso, conv_resi;
  double maxbo, residuo, err_u, err_p, err_t;
};

struct BCtl {
  int budget;      // outer iterations this launch may still run
  int any_active;
};

constexpr int kNorms = 5;  // dv, dp, bo, dT, residual

}  // namespace

struct ixb_batch {
  int count = 0, prec = 0;
  std::vector<ixb_handle*> h;
  cudaStream_t stream = nullptr;
  cudaError_t last_cuda = cudaSuccess;
  int nsm = 148;
  int tl[EQ_COUNT] = {}, g[EQ_COUNT] = {};
  // device tables (rebuilt when dirty)
  void* asm_inst[EQ_COUNT] = {};
  int2* asm_items[EQ_COUNT] = {};
  int asm_n[EQ_COUNT] = {};
  SolveInst* sol_inst[EQ_COUNT] = {};
  FusedInst* fus_inst[EQ_COUNT] = {};  // the same instances for the fused form (same work items)
  int2* sol_items[EQ_COUNT] = {};
  int sol_n[EQ_COUNT] = {};
  size_t sol_smem[EQ_COUNT] = {};
  CellInst* cell_inst = nullptr;
  int2* corr_items = nullptr;
  int2* res_items = nullptr;
  int ncorr = 0, nres = 0;
  // loop state
  int* active = nullptr;
  BInst* inst_d = nullptr;
  BInst* inst_h = nullptr;  // pinned
  BCtl* ctl_d = nullptr;
  BCtl* ctl_h = nullptr;    // pinned
  // norms: partials per work item, counters and results per instance
  double* partials[kNorms] = {};
  unsigned int* counters = nullptr;
  double* results = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool dirty = true;
  bool use_graph = true;  // IXB_NO_GRAPH=1: host-driven loop (one sync per iteration)
};

namespace {

#define BCK(x)                     \
  do {                             \
    cudaError_t e_ = (x);          \
    if (e_ != cudaSuccess) {       \
      b->last_cuda = e_;           \
      return IXB_ECUDA;            \
    }                              \
  } while (0)

#define BTRY(x)                    \
  do {                             \
    int s_ = (x);                  \
    if (s_ != IXB_OK) return s_;   \
  } while (0)

template <class T>
void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

void free_tables(ixb_batch* b) {
  for (int e = 0; e < EQ_COUNT; ++e) {
    dfree(b->asm_inst[e]); dfree(b->asm_items[e]); dfree(b->sol_inst[e]); dfree(b->sol_items[e]);
    dfree(b->fus_inst[e]);
  }
  dfree(b->cell_inst); dfree(b->corr_items); dfree(b->res_items);
  for (auto& p : b->partials) dfree(p);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

template <class T>
cudaError_t upload(T** dst, const std::vector<T>& v) {
  cudaError_t e = cudaMalloc((void**)dst, std::max<size_t>(1, v.size()) * sizeof(T));
  if (e != cudaSuccess) return e;
  return v.empty() ? cudaSuccess : cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

int form_of(const ixb_batch* b) { return b->prec == IXB_PREC_FP32_REFINED ? SOLVER_MIXED : IXB_SOLVER_HYBRID; }

// assembly descriptors of sweep EQ for every instance, typed for the form
template <int EQ, int SOLVER>
cudaError_t build_asm(ixb_batch* b, const std::vector<SweepIO<double>>& io, std::vector<int2>& items) {
  using ST = SweepTypes<SOLVER, EQ>;
  using S = typename ST::S;
  std::vector<AsmInst<S>> v(b->count);
  for (int i = 0; i < b->count; ++i) {
    ixb_handle* h = b->h[i];
    const SweepShape s = sweep_shape(EQ, h->mi, h->nj, (int)sizeof(S), 1, 128);
    AsmInst<S>& d = v[i];
    d.G = handle_geo(h);
    d.io = io[i];
    S* base = static_cast<S*>(h->stage);
    d.co.a = base; d.co.b = base + h->stage_stride; d.co.c = base + 2 * h->stage_stride;
    d.co.d = base + 3 * h->stage_stride; d.co.P = h->stage_P;
    d.n = s.n; d.line_lo = s.line_lo; d.line_hi = s.line_hi;
    d.first = (int)items.size();
    d.count = asm_tiles(EqIsX<EQ>::value, s.n, s.line_hi - s.line_lo + 1);
    for (int t = 0; t < d.count; ++t) items.push_back(make_int2(i, t));
  }
  AsmInst<S>* dv = nullptr;
  cudaError_t e = upload(&dv, v);
  b->asm_inst[EQ] = dv;
  return e;
}

template <int SOLVER>
cudaError_t build_asm_eq(ixb_batch* b, int eq, const std::vector<SweepIO<double>>& io, std::vector<int2>& items) {
  switch (eq) {
    case EQ_UY: return build_asm<EQ_UY, SOLVER>(b, io, items);
    case EQ_UX: return build_asm<EQ_UX, SOLVER>(b, io, items);
    case EQ_VY: return build_asm<EQ_VY, SOLVER>(b, io, items);
    case EQ_VX: return build_asm<EQ_VX, SOLVER>(b, io, items);
    case EQ_PY: return build_asm<EQ_PY, SOLVER>(b, io, items);
    case EQ_PX: return build_asm<EQ_PX, SOLVER>(b, io, items);
    case EQ_TY: return build_asm<EQ_TY, SOLVER>(b, io, items);
    default: return build_asm<EQ_TX, SOLVER>(b, io, items);
  }
}

template <int SOLVER>
cudaError_t launch_asm_eq(ixb_batch* b, int eq, const BatchNorm& bn) {
  const void* in = b->asm_inst[eq];
  const int2* it = b->asm_items[eq];
  const int n = b->asm_n[eq];
  switch (eq) {
    case EQ_UY: return assemble_batch_launch<EQ_UY, SOLVER>(in, it, n, b->active, bn, b->stream);
    case EQ_UX: return assemble_batch_launch<EQ_UX, SOLVER>(in, it, n, b->active, bn, b->stream);
    case EQ_VY: return assemble_batch_launch<EQ_VY, SOLVER>(in, it, n, b->active, bn, b->stream);
    case EQ_VX: return assemble_batch_launch<EQ_VX, SOLVER>(in, it, n, b->active, bn, b->stream);
    case EQ_PY: return assemble_batch_launch<EQ_PY, SOLVER>(in, it, n, b->active, bn, b->stream);
    case EQ_PX: return assemble_batch_launch<EQ_PX, SOLVER>(in, it, n, b->active, bn, b->stream);
    case EQ_TY: return assemble_batch_launch<EQ_TY, SOLVER>(in, it, n, b->active, bn, b->stream);
    default: return assemble_batch_launch<EQ_TX, SOLVER>(in, it, n, b->active, bn, b->stream);
  }
}

template <int SOLVER>
cudaError_t launch_fused_eq(ixb_batch* b, int eq, const BatchNorm& an, const BatchNorm& sn) {
  const int tl = b->tl[eq], g = b->g[eq];
  const size_t sm = b->sol_smem[eq];
  const FusedInst* in = b->fus_inst[eq];
  const int2* it = b->sol_items[eq];
  const int n = b->sol_n[eq];
  switch (eq) {
    case EQ_UY: return fused_batch_launch<EQ_UY, SOLVER>(tl, g, sm, in, it, n, b->active, an, sn, b->stream);
    case EQ_UX: return fused_batch_launch<EQ_UX, SOLVER>(tl, g, sm, in, it, n, b->active, an, sn, b->stream);
    case EQ_VY: return fused_batch_launch<EQ_VY, SOLVER>(tl, g, sm, in, it, n, b->active, an, sn, b->stream);
    case EQ_VX: return fused_batch_launch<EQ_VX, SOLVER>(tl, g, sm, in, it, n, b->active, an, sn, b->stream);
    case EQ_PY: return fused_batch_launch<EQ_PY, SOLVER>(tl, g, sm, in, it, n, b->active, an, sn, b->stream);
    case EQ_PX: return fused_batch_launch<EQ_PX, SOLVER>(tl, g, sm, in, it, n, b->active, an, sn, b->stream);
    case EQ_TY: return fused_batch_launch<EQ_TY, SOLVER>(tl, g, sm, in, it, n, b->active, an, sn, b->stream);
    default: return fused_batch_launch<EQ_TX, SOLVER>(tl, g, sm, in, it, n, b->active, an, sn, b->stream);
  }
}

// One sweep of every active instance: one fused launch where the shape has
// a fused form, else the assembly launch and the line-solve launch.  an:
// the b_o norm (p'-x), sn: the pass norm.
cudaError_t sweep_batch(ixb_batch* b, int eq, const BatchNorm& an, const BatchNorm& sn) {
  const int form = form_of(b);
  if (fused_enabled() && fused_shape(eq, b->tl[eq], b->g[eq])) {
    const cudaError_t e = form == SOLVER_MIXED ? launch_fused_eq<SOLVER_MIXED>(b, eq, an, sn)
                                               : launch_fused_eq<IXB_SOLVER_HYBRID>(b, eq, an, sn);
    if (e != cudaErrorNotSupported) return e;
  }
  cudaError_t e = form == SOLVER_MIXED ? launch_asm_eq<SOLVER_MIXED>(b, eq, an) : launch_asm_eq<IXB_SOLVER_HYBRID>(b, eq, an);
  if (e != cudaSuccess) return e;
  const bool dc = form == SOLVER_MIXED && eq != EQ_PY && eq != EQ_PX;
  return solve_batch_launch(form, (eq & 1) != 0, dc, b->tl[eq], b->g[eq], b->sol_smem[eq], b->sol_inst[eq],
                            b->sol_items[eq], b->sol_n[eq], b->active, sn, b->stream);
}

BatchNorm norm_of(ixb_batch* b, int k) {
  return BatchNorm{b->partials[k], b->counters + (size_t)k * b->count, b->results + (size_t)k * b->count};
}

// Descriptors and work items of one outer iteration for every instance
// (buffer parity 0 at the start of the iteration, back at 0 at its end).
int build_tables(ixb_batch* b) {
  free_tables(b);
  const int form = form_of(b);
  for (int eq = 0; eq < EQ_COUNT; ++eq) {
    if (b->tl[eq] == 0) {  // default line-solve shape: 2 lines x 64 threads
      b->tl[eq] = 2;
      b->g[eq] = 64;
    }
  }
  for (int i = 0; i < b->count; ++i) {
    ixb_handle* h = b->h[i];
    BTRY(handle_ready(h));
    BCK(cudaStreamSynchronize(h->stream));
    if (h->cu | h->cv | h->cT | h->cpc) return IXB_ESTATE;  // always 0 between outer iterations
  }
  // per-sweep io in the order of main.f90; p' starts each pass from zero
  std::vector<std::vector<SweepIO<double>>> io(EQ_COUNT, std::vector<SweepIO<double>>(b->count));
  for (int i = 0; i < b->count; ++i) {
    ixb_handle* h = b->h[i];
    io[EQ_UY][i] = handle_sweep_io(h, EQ_UY, nullptr);
    io[EQ_UX][i] = handle_sweep_io(h, EQ_UX, nullptr);
    const double* v_start = h->v[h->cv];
    io[EQ_VY][i] = handle_sweep_io(h, EQ_VY, nullptr);
    io[EQ_VX][i] = handle_sweep_io(h, EQ_VX, v_start);
    io[EQ_PY][i] = handle_sweep_io(h, EQ_PY, nullptr);
    io[EQ_PY][i].in = h->zero;
    io[EQ_PX][i] = handle_sweep_io(h, EQ_PX, h->zero);
    const double* t_start = h->T[h->cT];
    io[EQ_TY][i] = handle_sweep_io(h, EQ_TY, nullptr);
    io[EQ_TX][i] = handle_sweep_io(h, EQ_TX, t_start);
    if (h->cu | h->cv | h->cT | h->cpc) return IXB_ESTATE;
  }
  size_t max_items = 1;
  for (int eq = 0; eq < EQ_COUNT; ++eq) {
    std::vector<int2> items;
    cudaError_t e = form == SOLVER_MIXED ? build_asm_eq<SOLVER_MIXED>(b, eq, io[eq], items)
                                         : build_asm_eq<IXB_SOLVER_HYBRID>(b, eq, io[eq], items);
    BCK(e);
    BCK(upload(&b->asm_items[eq], items));
    b->asm_n[eq] = (int)items.size();
    max_items = std::max(max_items, items.size());
    // line solve: one shape (tl x g) for every instance
    std::vector<SolveInst> sv(b->count);
    std::vector<int2> sitems;
    size_t smem = 0;
    for (int i = 0; i < b->count; ++i) {
      ixb_handle* h = b->h[i];
      const SweepShape s = sweep_shape(eq, h->mi, h->nj, handle_real_bytes(h), b->tl[eq], b->g[eq]);
      SolveInst& d = sv[i];
      d.io.coef = h->stage; d.io.stride = h->stage_stride; d.io.P = h->stage_P;
      d.io.in = io[eq][i].in; d.io.out = io[eq][i].out; d.io.prev = io[eq][i].prev;
      d.io.LD = h->LD; d.io.m = s.m; d.io.mp = s.mp;
      d.n = s.n; d.line_lo = s.line_lo; d.line_hi = s.line_hi; d.nfull = s.nfull;
      d.first = (int)sitems.size();
      d.count = s.grid;
      for (int t = 0; t < s.grid; ++t) sitems.push_back(make_int2(i, t));
      smem = std::max(smem, s.smem);
    }
    BCK(upload(&b->sol_inst[eq], sv));
    std::vector<FusedInst> fv(b->count);
    for (int i = 0; i < b->count; ++i) fv[i] = FusedInst{handle_geo(b->h[i]), io[eq][i], sv[i]};
    BCK(upload(&b->fus_inst[eq], fv));
    BCK(upload(&b->sol_items[eq], sitems));
    b->sol_n[eq] = (int)sitems.size();
    b->sol_smem[eq] = smem;
    max_items = std::max(max_items, sitems.size());
  }
  // correction and residual
  std::vector<CellInst> cv(b->count);
  std::vector<int2> citems, ritems;
  for (int i = 0; i < b->count; ++i) {
    ixb_handle* h = b->h[i];
    CellInst& d = cv[i];
    d.G = handle_geo(h);
    d.u = h->u[0]; d.v = h->v[0]; d.p = h->p; d.resu = h->resu;
    d.pc = h->pc[0]; d.au = h->au; d.av = h->av; d.T = h->T[0]; d.u_ant = h->u_ant;
    d.fcon = h->fcon[0]; d.flin = h->flin[0];
    const int nc = ((h->mi - 1) * (h->nj - 1) + kCellChunk - 1) / kCellChunk;
    for (int t = 0; t < nc; ++t) citems.push_back(make_int2(i, t));
    d.first = (int)ritems.size();
    d.count = ((h->mi - 2) * (h->nj - 1) + kCellChunk - 1) / kCellChunk;
    for (int t = 0; t < d.count; ++t) ritems.push_back(make_int2(i, t));
  }
  BCK(upload(&b->cell_inst, cv));
  BCK(upload(&b->corr_items, citems));
  BCK(upload(&b->res_items, ritems));
  b->ncorr = (int)citems.size();
  b->nres = (int)ritems.size();
  max_items = std::max(max_items, ritems.size());
  for (auto& p : b->partials) BCK(cudaMalloc(&p, max_items * sizeof(double)));
  BCK(cudaMemset(b->counters, 0, (size_t)kNorms * b->count * sizeof(unsigned int)));
  return IXB_OK;
}

// one outer iteration of every active instance (main.f90:404-1215 with one
// pass of each inner loop)
int body(ixb_batch* b) {
  const int form = form_of(b);
  const BatchNorm none{nullptr, nullptr, nullptr};
  for (int eq = 0; eq < EQ_COUNT; ++eq) {
    const BatchNorm an = eq == EQ_PX ? norm_of(b, 2) : none;
    const BatchNorm sn = eq == EQ_VX ? norm_of(b, 0) : eq == EQ_PX ? norm_of(b, 1) : eq == EQ_TX ? norm_of(b, 3) : none;
    BCK(sweep_batch(b, eq, an, sn));
    if (eq == EQ_PX) BCK(correct_batch_launch(b->cell_inst, b->corr_items, b->ncorr, b->active, 1, b->stream));
  }
  BCK(residual_batch_launch(b->cell_inst, b->res_items, b->nres, b->active, norm_of(b, 4), 1, b->stream));
  return IXB_OK;
}

__device__ __forceinline__ bool finite_d(double x) { return isfinite(x); }

// After an outer iteration: the outer test of every active instance
// (main.f90:1202-1215), then the loop condition = any instance active and
// budget left.
__global__ void batch_ctl_kernel(BInst* inst, int* active, const double* results, int count, BCtl* ctl,
                                 cudaGraphConditionalHandle cond, int in_graph) {
  IXB_PDL_ENTRY();
  int any = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    if (!active[i]) continue;
    BInst& s = inst[i];
    s.iters++;
    s.err_u = results[0 * count + i];
    s.err_p = results[1 * count + i];
    s.maxbo = results[2 * count + i];
    s.err_t = results[3 * count + i];
    s.residuo = results[4 * count + i];
    if (!finite_d(s.maxbo) || !finite_d(s.residuo) || !finite_d(s.err_u) || !finite_d(s.err_t)) {
      s.status = IXB_ENONFINITE;
      s.exit_code = 3;
      active[i] = 0;
    } else if (s.maxbo < s.conv_paso && s.residuo < s.conv_resi) {
      s.exit_code = 1;
      active[i] = 0;
    } else {
      any = 1;
    }
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    ctl->budget -= 1;
    const bool go = any && ctl->budget > 0;
    if (!go)
      for (int i = 0; i < count; ++i)
        if (active[i] && inst[i].exit_code == 0) inst[i].exit_code = 2;
    ctl->any_active = go;
    if (in_graph) cudaGraphSetConditional(cond, go ? 1u : 0u);
  }
}

__global__ void batch_begin_kernel(const int* active, int count, BCtl* ctl, cudaGraphConditionalHandle cond) {
  IXB_PDL_ENTRY();
  int any = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) any |= active[i];
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) cudaGraphSetConditional(cond, (any && ctl->budget > 0) ? 1u : 0u);
}

int build_graph(ixb_batch* b) {
  cudaGraph_t g;
  BCK(cudaGraphCreate(&g, 0));
  b->graph = g;
  cudaGraphConditionalHandle cond;
  BCK(cudaGraphConditionalHandleCreate(&cond, g, 0, 0));
  // begin: condition from the active flags and the budget
  cudaGraphNode_t n_begin, n_while;
  {
    BCK(cudaStreamBeginCaptureToGraph(b->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const cudaError_t le = launch_k(batch_begin_kernel, 1, 256, 0, b->stream, (const int*)b->active, b->count, b->ctl_d, cond);
    cudaGraph_t out = nullptr;
    BCK(cudaStreamEndCapture(b->stream, &out));
    BCK(le);
    size_t nn = 1;
    BCK(cudaGraphGetNodes(g, &n_begin, &nn));
    if (nn != 1) return IXB_ECUDA;
  }
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = cond;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  BCK(cudaGraphAddNode(&n_while, g, &n_begin, 1, &wp));
  cudaGraph_t bodyg = wp.conditional.phGraph_out[0];
  BCK(cudaStreamBeginCaptureToGraph(b->stream, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  int st = body(b);
  if (st == IXB_OK) {
    if (launch_k(batch_ctl_kernel, 1, 256, 0, b->stream, b->inst_d, b->active, (const double*)b->results, b->count,
                 b->ctl_d, cond, 1) != cudaSuccess)
      st = IXB_ECUDA;
  }
  cudaGraph_t captured;
  const cudaError_t ce = cudaStreamEndCapture(b->stream, &captured);
  if (st != IXB_OK) return st;
  BCK(ce);
  BCK(cudaGraphInstantiate(&b->exec, g, 0));
  return IXB_OK;
}

int ensure_ready(ixb_batch* b) {
  if (!b->dirty && (b->exec || !b->use_graph)) return IXB_OK;
  BTRY(build_tables(b));
  if (b->use_graph) BTRY(build_graph(b));
  b->dirty = false;
  return IXB_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int ixb_batch_create(int count, const int* mi, const int* nj, int prec_mode, ixb_batch** out) {
  if (!out || count < 1 || !mi || !nj) return IXB_EINVAL;
  *out = nullptr;
  if (prec_mode != IXB_PREC_FP64 && prec_mode != IXB_PREC_FP32_REFINED) return IXB_EINVAL;
  for (int i = 0; i < count; ++i)
    if (mi[i] < 4 || nj[i] < 4 || mi[i] > 1024 || nj[i] > 1024) return IXB_EINVAL;
  ixb_batch* b = new (std::nothrow) ixb_batch();
  if (!b) return IXB_ENOMEM;
  b->count = count;
  b->prec = prec_mode;
  b->h.assign(count, nullptr);
  auto fail = [&](int code) { ixb_batch_destroy(b); return code; };
  for (int i = 0; i < count; ++i) {
    const int st = ixb_create(mi[i], nj[i], prec_mode, &b->h[i]);
    if (st != IXB_OK) return fail(st);
  }
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(IXB_ECUDA);
  if (cudaMalloc(&b->active, count * sizeof(int)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMalloc(&b->inst_d, count * sizeof(BInst)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMallocHost(&b->inst_h, count * sizeof(BInst)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMalloc(&b->ctl_d, sizeof(BCtl)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMallocHost(&b->ctl_h, sizeof(BCtl)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMalloc(&b->counters, (size_t)kNorms * count * sizeof(unsigned int)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMalloc(&b->results, (size_t)kNorms * count * sizeof(double)) != cudaSuccess) return fail(IXB_ENOMEM);
  if (cudaMemset(b->active, 0, count * sizeof(int)) != cudaSuccess) return fail(IXB_ECUDA);
  if (cudaMemset(b->results, 0, (size_t)kNorms * count * sizeof(double)) != cudaSuccess) return fail(IXB_ECUDA);
  std::memset(b->inst_h, 0, count * sizeof(BInst));
  if (cudaMemcpy(b->inst_d, b->inst_h, count * sizeof(BInst), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(IXB_ECUDA);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return fail(IXB_ECUDA);
  const char* env = std::getenv("IXB_NO_GRAPH");
  if (env && env[0] == '1') b->use_graph = false;
  *out = b;
  return IXB_OK;
}

int ixb_batch_destroy(ixb_batch* b) {
  if (!b) return IXB_EINVAL;
  if (b->stream) cudaStreamSynchronize(b->stream);
  free_tables(b);
  dfree(b->active); dfree(b->inst_d); dfree(b->ctl_d); dfree(b->counters); dfree(b->results);
  if (b->inst_h) cudaFreeHost(b->inst_h);
  if (b->ctl_h) cudaFreeHost(b->ctl_h);
  for (ixb_handle* h : b->h)
    if (h) ixb_destroy(h);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return IXB_OK;
}

int ixb_batch_instance(ixb_batch* b, int i, ixb_handle** h) {
  if (!b || !h || i < 0 || i >= b->count) return IXB_EINVAL;
  *h = b->h[i];
  b->dirty = true;  // the caller may change mesh, parameters or boundary tables through it
  return IXB_OK;
}

int ixb_batch_set_sweep_shape(ixb_batch* b, int sweep, int lines_per_cta, int threads_per_line) {
  if (!b || sweep < 0 || sweep >= EQ_COUNT) return IXB_EINVAL;
  const auto& shapes = kShapeList;
  bool ok = lines_per_cta == 0;
  for (auto& s : shapes) ok |= (s[0] == lines_per_cta && s[1] == threads_per_line);
  if (!ok) return IXB_EINVAL;
  b->tl[sweep] = lines_per_cta;
  b->g[sweep] = threads_per_line;
  b->dirty = true;
  return IXB_OK;
}

int ixb_batch_autotune(ixb_batch* b, int reps, int* chosen, double* ms) {
  if (!b || reps < 1) return IXB_EINVAL;
  const auto& shapes = kShapeList;
  for (ixb_handle* h : b->h) BCK(cudaStreamSynchronize(h->stream));
  // every buffer a sweep may write, saved and restored around the trials
  std::vector<std::pair<double*, double*>> saved;
  size_t total = 0;
  for (ixb_handle* h : b->h) total += 11 * h->fsz;
  double* pool = nullptr;
  BCK(cudaMalloc(&pool, total * sizeof(double)));
  std::vector<int> act(b->count);
  BCK(cudaMemcpy(act.data(), b->active, b->count * sizeof(int), cudaMemcpyDeviceToHost));
  std::vector<int> on(b->count, 1);
  BCK(cudaMemcpy(b->active, on.data(), b->count * sizeof(int), cudaMemcpyHostToDevice));
  size_t off = 0;
  for (ixb_handle* h : b->h) {
    double* bufs[11] = {h->u[0], h->u[1], h->v[0], h->v[1], h->T[0], h->T[1], h->pc[0], h->pc[1], h->au, h->av, h->b_o};
    for (double* p : bufs) {
      BCK(cudaMemcpyAsync(pool + off, p, h->fsz * sizeof(double), cudaMemcpyDeviceToDevice, b->stream));
      saved.emplace_back(p, pool + off);
      off += h->fsz;
    }
  }
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0));
  BCK(cudaEventCreate(&e1));
  const int form = form_of(b);
  const BatchNorm none{nullptr, nullptr, nullptr};
  int st = IXB_OK;
  for (int eq = 0; eq < EQ_COUNT && st == IXB_OK; ++eq) {
    double best = 1e300;
    int bk = -1;
    for (int k = 0; k < kNumShapes && st == IXB_OK; ++k) {
      b->tl[eq] = shapes[k][0];
      b->g[eq] = shapes[k][1];
      if ((st = build_tables(b)) != IXB_OK) break;
      auto once = [&]() -> cudaError_t { return sweep_batch(b, eq, none, none); };
      cudaError_t e = once();
      if (e == cudaErrorInvalidValue) { cudaGetLastError(); continue; }  // shape cannot run here
      if (e != cudaSuccess) { b->last_cuda = e; st = IXB_ECUDA; break; }
      cudaEventRecord(e0, b->stream);
      for (int r = 0; r < reps && e == cudaSuccess; ++r) e = once();
      cudaEventRecord(e1, b->stream);
      if (e != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) { b->last_cuda = e; st = IXB_ECUDA; break; }
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      if (t / reps < best) { best = t / reps; bk = k; }
    }
    if (st != IXB_OK) break;
    if (bk < 0) { st = IXB_EINVAL; break; }
    b->tl[eq] = shapes[bk][0];
    b->g[eq] = shapes[bk][1];
    if (chosen) { chosen[2 * eq] = b->tl[eq]; chosen[2 * eq + 1] = b->g[eq]; }
    if (ms) ms[eq] = best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  off = 0;
  for (ixb_handle* h : b->h) {
    for (int q = 0; q < 11; ++q) {
      auto& pr = saved[off++];
      cudaMemcpyAsync(pr.first, pr.second, h->fsz * sizeof(double), cudaMemcpyDeviceToDevice, b->stream);
    }
  }
  cudaMemcpyAsync(b->active, act.data(), b->count * sizeof(int), cudaMemcpyHostToDevice, b->stream);
  const cudaError_t se = cudaStreamSynchronize(b->stream);
  cudaFree(pool);
  b->dirty = true;
  if (st != IXB_OK) return st;
  BCK(se);
  return IXB_OK;
}

int ixb_batch_restart(ixb_batch* b) {
  if (!b) return IXB_EINVAL;
  for (int i = 0; i < b->count; ++i) {
    ixb_handle* h = b->h[i];
    BInst& s = b->inst_h[i];
    std::memset(&s, 0, sizeof(BInst));
    s.conv_paso = h->prm.conv_paso;
    s.conv_resi = h->prm.conv_resi;
  }
  BCK(cudaMemcpyAsync(b->inst_d, b->inst_h, b->count * sizeof(BInst), cudaMemcpyHostToDevice, b->stream));
  std::vector<int> on(b->count, 1);
  BCK(cudaMemcpyAsync(b->active, on.data(), b->count * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return IXB_OK;
}

int ixb_batch_iterate(ixb_batch* b, int max_iters, int* n_active) {
  if (!b || max_iters < 0) return IXB_EINVAL;
  for (ixb_handle* h : b->h) BCK(cudaStreamSynchronize(h->stream));
  BTRY(ensure_ready(b));
  b->ctl_h->budget = max_iters;
  b->ctl_h->any_active = 0;
  BCK(cudaMemcpyAsync(b->ctl_d, b->ctl_h, sizeof(BCtl), cudaMemcpyHostToDevice, b->stream));
  if (max_iters > 0 && b->use_graph) BCK(cudaGraphLaunch(b->exec, b->stream));
  if (max_iters > 0 && !b->use_graph) {  // the same kernels driven from the host
    for (;;) {
      BTRY(body(b));
      BCK(launch_k(batch_ctl_kernel, 1, 256, 0, b->stream, b->inst_d, b->active, (const double*)b->results, b->count,
                   b->ctl_d, cudaGraphConditionalHandle{}, 0));
      BCK(cudaMemcpyAsync(b->ctl_h, b->ctl_d, sizeof(BCtl), cudaMemcpyDeviceToHost, b->stream));
      BCK(cudaStreamSynchronize(b->stream));
      if (!b->ctl_h->any_active) break;
    }
  }
  BCK(cudaMemcpyAsync(b->inst_h, b->inst_d, b->count * sizeof(BInst), cudaMemcpyDeviceToHost, b->stream));
  std::vector<int> act(b->count);
  BCK(cudaMemcpyAsync(act.data(), b->active, b->count * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  int n = 0;
  for (int a : act) n += a != 0;
  if (n_active) *n_active = n;
  return IXB_OK;
}

int ixb_batch_report(ixb_batch* b, int i, ixb_report* out) {
  if (!b || !out || i < 0 || i >= b->count) return IXB_EINVAL;
  const BInst& s = b->inst_h[i];
  std::memset(out, 0, sizeof(*out));
  out->maxbo = s.maxbo;
  out->residuo = s.residuo;
  out->err_u = s.err_u;
  out->err_p = s.err_p;
  out->err_t = s.err_t;
  out->n_simple = s.iters;
  out->n_momen = out->n_pres = out->n_ener = s.iters;
  out->exit_code = s.exit_code;
  out->status = s.status;
  return IXB_OK;
}

}  // extern "C"
