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
// Returns whether the loop runs another pass.
static __device__ bool ctl_inner_step(Ctl* c, const double* norms, int which, cudaGraphConditionalHandle inner) {
  double err, conv;
  if (which == 0) { err = norms[N_DV]; conv = c->conv_u; c->err_u = err; c->n_momen++; }
  else if (which == 1) { err = norms[N_DP]; conv = c->conv_p; c->err_p = err; c->maxbo = norms[N_BO]; c->n_pres++; }
  else { err = norms[N_DT]; conv = c->conv_t; c->err_t = err; c->n_ener++; }
  bool again;
  c->inner_done++;
  if (!finite_d(err) || (which == 1 && !finite_d(norms[N_BO]))) {
    c->status = IXB_ENONFINITE;  // the outer control ends the loop
    again = false;
  } else if (err < conv) { c->iter_ecuaci = 0; again = false; }
  else if (c->iter_ecuaci > c->iter_ecuaci_max) { c->iter_ecuaci = 0; again = false; }
  else { c->iter_ecuaci++; again = true; }
  // the reference's counter logic bounds a loop by iter_ecuaci_max + 2
  // passes; enforce it independently so no WHILE node can run away
  if (again && (long long)c->inner_done >= (long long)c->iter_ecuaci_max + 2) { c->status = IXB_ETIMEOUT; again = false; }
  if (!again) c->inner_done = 0;  // the next inner loop counts from zero
  cudaGraphSetConditional(inner, again ? 1u : 0u);
  return again;
}

// Start of an inner loop: after a non-finite stop, the later inner loops of
// the same outer pass must not run.
static __device__ void ctl_gate_step(Ctl* c, cudaGraphConditionalHandle inner) {
  cudaGraphSetConditional(inner, c->status == 0 ? 1u : 0u);
}

// End of an outer pass; also opens the momentum loop of the next pass.
static __device__ void ctl_outer_step(Ctl* c, const double* norms, cudaGraphConditionalHandle outer,
                                      cudaGraphConditionalHandle first_inner) {
  c->inner_done = 0;
  cudaGraphSetConditional(first_inner, 1u);
  if (c->status != 0) { cudaGraphSetConditional(outer, 0); return; }
  c->residuo = norms[N_RES];
  c->n_simple++;
  c->outer_done++;
  if (!finite_d(c->residuo)) { c->status = IXB_ENONFINITE; cudaGraphSetConditional(outer, 0); return; }
  if (c->fixed_count > 0) {
    cudaGraphSetConditional(outer, c->outer_done < c->fixed_count ? 1u : 0u);
    return;
  }
  bool again;
  if (c->maxbo < c->conv_paso && c->residuo < c->conv_resi) { c->iter_simple = 0; c->exit_code = 1; again = false; }
  else if (c->iter_simple > c->iter_simple_max) { c->iter_simple = 0; c->exit_code = 2; again = false; }
  else { c->iter_simple++; again = true; }
  if (again && (long long)c->outer_done >= (long long)c->iter_simple_max + 2) { c->status = IXB_ETIMEOUT; again = false; }
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
