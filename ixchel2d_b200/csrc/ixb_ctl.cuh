// ixb_ctl.cuh -- the device-side loop control of the graph-driven SIMPLE
// loop: the reference's inner-loop exit tests (source/main.f90:729-740,
// :913-924, :1144-1156) and outer test (:1202-1215), run by one thread of
// the kernel that finishes the norm they read, which then sets the loop's
// conditional graph node.
#pragma once
#include <cuda_runtime.h>

#include "ixb_handle.h"

namespace ixb {

__device__ __forceinline__ bool finite_d(double x) { return isfinite(x); }

// End of an inner pass.  which: 0 momentum (||dv|| vs conv_u), 1 pressure
// (||dp'|| vs conv_p, with maxbo), 2 energy (||dT|| vs conv_t).
// Returns whether the loop runs another pass.  Every field is loaded before
// any is stored (one round trip to memory instead of a chain of them: a
// store to the control block would otherwise order the loads after it).
static __device__ bool ctl_inner_step(Ctl* c, const double* norms, int which, cudaGraphConditionalHandle inner) {
  const double n_dv = norms[N_DV], n_dp = norms[N_DP], n_bo = norms[N_BO], n_dt = norms[N_DT];
  const double conv_u = c->conv_u, conv_p = c->conv_p, conv_t = c->conv_t;
  const int iter = c->iter_ecuaci, iter_max = c->iter_ecuaci_max, done = c->inner_done + 1;
  const long long n_momen = c->n_momen, n_pres = c->n_pres, n_ener = c->n_ener;
  const double err = which == 0 ? n_dv : (which == 1 ? n_dp : n_dt);
  const double conv = which == 0 ? conv_u : (which == 1 ? conv_p : conv_t);
  bool again;
  int status = 0, iter_new = iter;
  if (!finite_d(err) || (which == 1 && !finite_d(n_bo))) {
    status = IXB_ENONFINITE;  // the outer control ends the loop
    again = false;
  } else if (err < conv) { iter_new = 0; again = false; }
  else if (iter > iter_max) { iter_new = 0; again = false; }
  else { iter_new = iter + 1; again = true; }
  // the reference's counter logic bounds a loop by iter_ecuaci_max + 2
  // passes; enforce it independently so no WHILE node can run away
  if (again && (long long)done >= (long long)iter_max + 2) { status = IXB_ETIMEOUT; again = false; }
  if (which == 0) { c->err_u = err; c->n_momen = n_momen + 1; }
  else if (which == 1) { c->err_p = err; c->maxbo = n_bo; c->n_pres = n_pres + 1; }
  else { c->err_t = err; c->n_ener = n_ener + 1; }
  if (status != 0) c->status = status;
  c->iter_ecuaci = iter_new;
  c->inner_done = again ? done : 0;  // the next inner loop counts from zero
  cudaGraphSetConditional(inner, again ? 1u : 0u);
  return again;
}

// Start of an inner loop: after a non-finite stop, the later inner loops of
// the same outer pass must not run.
static __device__ void ctl_gate_step(Ctl* c, cudaGraphConditionalHandle inner) {
  cudaGraphSetConditional(inner, c->status == 0 ? 1u : 0u);
}

// End of an outer pass; also opens the momentum loop of the next pass.
// Loads first, then stores, as in ctl_inner_step.
static __device__ void ctl_outer_step(Ctl* c, const double* norms, cudaGraphConditionalHandle outer,
                                      cudaGraphConditionalHandle first_inner) {
  const int status = c->status, fixed = c->fixed_count, done = c->outer_done + 1;
  const int iter = c->iter_simple, iter_max = c->iter_simple_max;
  const long long n_simple = c->n_simple;
  const double res = norms[N_RES], maxbo = c->maxbo, conv_paso = c->conv_paso, conv_resi = c->conv_resi;
  c->inner_done = 0;
  cudaGraphSetConditional(first_inner, 1u);
  if (status != 0) { cudaGraphSetConditional(outer, 0); return; }
  c->residuo = res;
  c->n_simple = n_simple + 1;
  c->outer_done = done;
  if (!finite_d(res)) { c->status = IXB_ENONFINITE; cudaGraphSetConditional(outer, 0); return; }
  if (fixed > 0) {
    cudaGraphSetConditional(outer, done < fixed ? 1u : 0u);
    return;
  }
  bool again;
  if (maxbo < conv_paso && res < conv_resi) { c->iter_simple = 0; c->exit_code = 1; again = false; }
  else if (iter > iter_max) { c->iter_simple = 0; c->exit_code = 2; again = false; }
  else { c->iter_simple = iter + 1; again = true; }
  if (again && (long long)done >= (long long)iter_max + 2) { c->status = IXB_ETIMEOUT; again = false; }
  cudaGraphSetConditional(outer, again ? 1u : 0u);
}

// After a block of outer passes of ixb_simple_converge: record the Nusselt
// numbers of both walls (nu2) and |Nu - Nu at the previous evaluation| of the
// monitored wall, then stop the monitor loop (exit_code 3) when that change
// is below mon_tol_dnu, (4) when maxbo is below mon_tol_maxbo, (5) once
// mon_max_iters outer passes are done, or on an error status of the passes.
static __device__ void ctl_monitor_step(Ctl* c, const double* nu2, cudaGraphConditionalHandle mon) {
  c->mon_nu[0] = nu2[0];
  c->mon_nu[1] = nu2[1];
  const double nu = nu2[c->mon_wall];
  const double dnu = c->mon_evals > 0 ? fabs(nu - c->mon_nu_prev) : INFINITY;
  c->mon_dnu = dnu;
  c->mon_nu_prev = nu;
  c->mon_evals++;
  bool stop = true;
  if (c->status != 0) {
  } else if (!finite_d(nu)) {
    c->status = IXB_ENONFINITE;
  } else if (dnu < c->mon_tol_dnu) {
    c->exit_code = 3;
  } else if (c->maxbo < c->mon_tol_maxbo) {
    c->exit_code = 4;
  } else if (c->n_simple >= c->mon_max_iters) {
    c->exit_code = 5;
  } else {
    stop = false;
  }
  cudaGraphSetConditional(mon, stop ? 0u : 1u);
}

}  // namespace ixb
