// ixb_handle.h -- the handle behind the C ABI (one SIMPLE instance on one
// CUDA stream), shared by the single-instance driver (ixb_api.cu) and the
// batched driver (ixb_batch.cu).  Not part of the public ABI.
#pragma once
#include <functional>
#include <cuda_runtime.h>

#include <vector>

#include "ixb_internal.h"

namespace ixb {

// device-side loop state for the graph-driven SIMPLE loop
struct Ctl {
  // inputs
  double conv_u, conv_p, conv_t, conv_resi, conv_paso;
  int iter_ecuaci_max, iter_simple_max;
  int fixed_count;   // >0: run exactly this many outer passes, no outer test
  // state
  int iter_ecuaci, iter_simple;
  int outer_done;    // passes done in this launch (in a monitor block: in this block)
  int inner_done;    // passes of the current inner loop (hard cap: iter_ecuaci_max + 2)
  int exit_code, status;
  long long n_simple, n_momen, n_pres, n_ener;
  double err_u, err_p, err_t, maxbo, residuo;
  // Nusselt monitor (ixb_simple_converge): inputs
  int mon_vertical, mon_k0, mon_k1, mon_wall;
  long long mon_max_iters;
  double mon_tol_dnu, mon_tol_maxbo;
  // Nusselt monitor: state
  long long mon_evals;
  double mon_nu[2], mon_nu_prev, mon_dnu;
};

// the SIMPLE loop graphs of a handle
enum GraphKind { GRAPH_PLAIN = 0, GRAPH_UNROLLED = 1, GRAPH_MON_PLAIN = 2, GRAPH_MON_UNROLLED = 3 };

}  // namespace ixb

struct ixb_handle {
  int mi = 0, nj = 0, LD = 0, rows = 0, prec = 0;
  size_t fsz = 0;  // elements per field buffer
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaError_t last_cuda = cudaSuccess;
  // fields (binary64)
  double *u[2] = {}, *v[2] = {}, *T[2] = {}, *pc[2] = {};
  double *p = nullptr, *u_ant = nullptr, *v_ant = nullptr, *T_ant = nullptr;
  double *au = nullptr, *av = nullptr, *b_o = nullptr, *resu = nullptr;
  double *fcon[3] = {}, *flin[3] = {};
  double* zero = nullptr;  // a field of zeros: the sources of an equation without any
  // rows of one sweep staged between its assembly and its line solve
  void* stage = nullptr;
  size_t stage_stride = 0;  // elements per row array
  int stage_P = 0;          // row pitch of a line
  int cu = 0, cv = 0, cT = 0, cpc = 0;
  // mesh
  double* metrics = nullptr;
  int mstride = 0;
  double* tables = nullptr;  // T_COUNT mesh-constant 2-D tables
  bool tables_dirty = true;
  double *xp_d = nullptr, *yp_d = nullptr;
  std::vector<double> xu, yv, xp, yp;
  // boundary tables [var][side][line]
  ixb::BCEntry* bc = nullptr;
  int bcstride = 0;
  // reductions
  double* partials = nullptr;
  unsigned int* counters = nullptr;
  double* norms = nullptr;
  int pstride = 0;
  double* h_norms = nullptr;  // pinned
  double* nu_d = nullptr;
  // control for graphs
  ixb::Ctl* ctl_d = nullptr;
  ixb::Ctl* ctl_h = nullptr;  // pinned
  bool graph_dirty = true;  // set by every change that invalidates the SIMPLE graphs
  // the SIMPLE loop graphs, by kind (ixb::GraphKind): the plain loop, the
  // same loop with kOuterUnroll outer passes per WHILE body for fixed counts
  // (ixb_simple_iterations), and both of those inside the Nusselt monitor's
  // WHILE loop (ixb_simple_converge)
  cudaGraph_t graphs[4] = {};
  cudaGraphExec_t graph_execs[4] = {};
  bool graph_stale[4] = {true, true, true, true};
  // K passes of the energy sweeps (ixb_energy_iterations) and of the energy
  // adjoint's reversed sweeps (ixb_adjoint_energy): WHILE graphs whose
  // counter kernel closes the loop after `loop_left` passes
  cudaGraphExec_t egraph_exec = nullptr, agraph_exec = nullptr;
  cudaGraph_t egraph = nullptr, agraph = nullptr;
  bool egraph_dirty = true, agraph_dirty = true;
  const double* agraph_pool = nullptr;  // adj_pool the adjoint graph was built on
  int* loop_left = nullptr;
  // params and flags
  ixb_params prm{};
  bool has_mesh = false, has_params = false, has_bc[3] = {false, false, false};
  int iter_ecuaci = 0, iter_simple = 0;
  int use_graph = 1;
  int shape_tl[ixb::EQ_COUNT] = {};  // launch shape per sweep (0 = not chosen yet)
  int shape_g[ixb::EQ_COUNT] = {};
  int nsm = 148;
  // adjoint workspace (ixb_adjoint_energy), allocated on first use
  double* xfer = nullptr;  // seven host-shaped (column-major, unpadded) state arrays: the state transfers' staging, allocated on the first transfer
  // asynchronous downloads (ixb_download_state_async): a snapshot of the
  // state in host layout, copied to the host on a stream of its own
  double* snap = nullptr;
  cudaStream_t dl_stream = nullptr;
  cudaEvent_t snap_ev = nullptr, dl_ev = nullptr;
  bool dl_pending = false;
  double* adj_pool = nullptr;
  size_t adj_size = 0;
};

namespace ixb {
// views and state of a handle used by the batched driver (defined in ixb_api.cu)
Geo<double> handle_geo(const ixb_handle* h);
int handle_solver_form(const ixb_handle* h);
int handle_ready(ixb_handle* h);  // mesh, params and boundary tables set; mesh tables built
// inputs/outputs of sweep `eq` at the current buffer parity (flips it), no norms
// WHILE graph whose body runs `pass` (launches on the handle's stream that
// leave buffer parity unchanged) `unroll` times, then a counter: built once,
// run by handle_run_loop_graph(h, exec, iterations) (stream-ordered,
// iterations >= 1; unroll * iterations passes)
constexpr int kLoopUnroll = 10;
// outer SIMPLE passes per WHILE body in the fixed-count graph
constexpr int kOuterUnroll = 4;
int handle_build_loop_graph(ixb_handle* h, const std::function<int()>& pass, int unroll, cudaGraph_t* graph,
                            cudaGraphExec_t* exec);
int handle_run_loop_graph(ixb_handle* h, cudaGraphExec_t exec, int iterations);
SweepIO<double> handle_sweep_io(ixb_handle* h, int eq, const double* prev);
int handle_real_bytes(const ixb_handle* h);  // element size of the staged rows
}  // namespace ixb
