/*
 * ixb.h -- C ABI of libixb, the B200 (sm_100a) SIMPLE outer iteration of
 * Ixchel2D.
 *
 * The reference has no C ABI: its hot path is Fortran module state plus
 * per-cell `!$acc routine` subroutines called from PROGRAM IXCHEL2D
 * (source/main.f90:395-1217).  Each entry point below names the reference
 * code it replaces.  All functions return an int status (IXB_OK = 0).
 * Calls on one handle are not thread-safe; separate handles are independent
 * (each owns its own device memory and CUDA stream).
 *
 * Array convention (host side): every 2-D array is Fortran column-major
 * with the reference's shapes, index (ii,jj) at (jj-1)*rows + (ii-1):
 *   u, u_ant, au, Resu, fuente_*_u   (mi,   nj+1)
 *   v, v_ant, av, fuente_*_v         (mi+1, nj  )
 *   p, T, T_ant, corr_pres, b_o, fuente_*_t  (mi+1, nj+1)
 * Mesh vectors: xu(mi), yv(nj), xp(mi+1), yp(nj+1).
 */
#ifndef IXB_H
#define IXB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define IXB_OK 0
#define IXB_EINVAL 1     /* bad argument (NULL handle, size out of range, ...) */
#define IXB_ECUDA 2      /* a CUDA runtime call failed */
#define IXB_ENONFINITE 3 /* a convergence norm became NaN or Inf */
#define IXB_ETIMEOUT 4   /* a bounded device wait expired */
#define IXB_EBC 5        /* a boundary table leaves a solved line without a row */
#define IXB_ESTATE 6     /* call order: mesh/params/bc not set yet */
#define IXB_EIO 7        /* file could not be read / parsed / written */
#define IXB_ENOMEM 8     /* device or host allocation failed */

/* precision modes for ixb_create.  Fields are held in binary64 in both.
 * IXB_PREC_FP32_REFINED (with IXB_SOLVER_HYBRID): every row is assembled in
 * binary64, scaled to a unit diagonal, and its line staged and solved in
 * binary32.  The u, v and T sweeps are defect corrections: the residual
 * d - A x of the current values is evaluated in binary64, the correction is
 * solved for in binary32 and added back in binary64, so the converged fields
 * are the binary64 ones.  The p' lines are solved outright in binary32 around
 * a binary64 mass source b_o; the p update and the convergence norms stay in
 * binary64.
 * IXB_SOLVER_EXACT ignores the mode and runs the binary64 reference order. */
#define IXB_PREC_FP64 0
#define IXB_PREC_FP32_REFINED 1

/* line solvers */
#define IXB_SOLVER_HYBRID 0 /* warp Thomas-PCR hybrid (default, fast) */
#define IXB_SOLVER_EXACT 1  /* sequential Thomas, bit-identical to
                               source/mod_solucionador.f90:25-47 */

/* variables for ixb_set_bc / ixb_set_sources */
#define IXB_VAR_U 0
#define IXB_VAR_V 1
#define IXB_VAR_T 2

/* boundary-segment types (tipo_condi strings of source/mod_cond_frontera.f90:34) */
#define IXB_BC_OTHER 0 /* any string other than 'diri'/'neum' (e.g. the default 'desc') */
#define IXB_BC_DIRI 1
#define IXB_BC_NEUM 2

typedef struct ixb_handle ixb_handle;

/* Solver parameters: the numeric records of parametros.dat after the
 * non-dimensionalisation of source/main.f90:221-244. */
typedef struct {
  double gamma_momen;  /* sqrt(Pr/Ra) natural, 1/Re mixed            */
  double gamma_energ;  /* sqrt(1/(Pr*Ra)) natural, 1/(Re*Pr) mixed   */
  double Ri;           /* u-momentum buoyancy coefficient (0 in both modes) */
  double Riy;          /* v-momentum buoyancy coefficient (-1 natural, Ri mixed) */
  double dt;
  double rel_vel, rel_pres, rel_ener;
  double conv_u, conv_p, conv_t, conv_resi, conv_paso;
  double p_update;     /* pressure under-relaxation, 0.6 in the reference (main.f90:934) */
  int iter_ecuaci_max;
  int iter_simple_max;
  int solver;          /* IXB_SOLVER_* */
  int reserved[5];
} ixb_params;

/* One side of tipo_cond_front (source/mod_cond_frontera.f90:25-38) after
 * lectura_cond_frontera: `index` holds indice_div(1..ndivis+1), 1-based.
 * (The reference declares indice_div(14); 16 entries let 15 divisions fit.) */
typedef struct {
  int side;         /* 0..3 = 'a','b','c','d' */
  int ndivis;       /* 0..15 */
  int type[15];     /* IXB_BC_* */
  double value[15];
  int index[16];
} ixb_bc_side;

/* Outcome of a SIMPLE call. */
typedef struct {
  double maxbo;     /* ||b_o||_2 of the last pressure pass (main.f90:898-906) */
  double residuo;   /* ||Resu||_2 of the last outer iteration (main.f90:1192-1199) */
  double err_u, err_p, err_t; /* last inner-loop errors (||dv||, ||dp'||, ||dT||) */
  int64_t n_simple; /* outer iterations run in this call */
  int64_t n_momen, n_pres, n_ener; /* inner passes run in this call */
  int exit_code;    /* 0 none (fixed count), 1 converged, 2 iteration limit;
                       ixb_simple_converge: 3 |dNu| below tol_dnu, 4 maxbo below
                       tol_maxbo, 5 max_iters reached */
  int status;
} ixb_report;

/* ---- library ---- */
int ixb_version(void);
const char* ixb_strerror(int status);
/* Number of CUDA devices visible (0 on a host without a GPU). */
int ixb_device_count(void);

/* ---- handle lifetime: replaces the `!$acc data` region of main.f90:356-389 ---- */
/* mi, nj: the grid sizes of source/mod_malla.f90:15, here chosen at run time
 * (4 <= mi, nj <= 6000). */
int ixb_create(int mi, int nj, int prec_mode, ixb_handle** out);
int ixb_destroy(ixb_handle* h);
/* Use an external CUDA stream (cudaStream_t) instead of the handle's own. */
int ixb_set_stream(ixb_handle* h, void* stream);

/* ---- inputs ---- */
/* Mesh coordinates; the metrics delta*, fe* are derived exactly as in
 * lectura_mallas_escalonadas (source/mod_malla.f90:167-218). */
int ixb_set_mesh(ixb_handle* h, const double* xu, const double* yv, const double* xp, const double* yp);
int ixb_set_params(ixb_handle* h, const ixb_params* p);
/* Boundary tables for u, v or T (the cond_front_* structures of
 * source/mod_ec_momento.f90:46-47, mod_ec_energia.f90:34) as applied by
 * impone_cond_frontera (source/mod_cond_frontera.f90:254-420).  Returns
 * IXB_EBC when a line that the reference solves would be left without a
 * boundary row (the reference would then read stale coefficients). */
int ixb_set_bc(ixb_handle* h, int var, const ixb_bc_side sides[4]);
/* Source terms fuente_con_*, fuente_lin_* (source/mod_ec_momento.f90:34-35,
 * mod_ec_energia.f90:30), e.g. immersed-body masks (mod_front_inmersa.f90:54-179).
 * NULL arrays mean zero. */
int ixb_set_sources(ixb_handle* h, int var, const double* fuente_con, const double* fuente_lin);

/* ---- state transfer (host arrays, Fortran shapes); NULL pointers are skipped ---- */
int ixb_upload_state(ixb_handle* h, const double* u, const double* v, const double* p, const double* T,
                     const double* u_ant, const double* v_ant, const double* T_ant);
int ixb_download_state(ixb_handle* h, double* u, double* v, double* p, double* T, double* u_ant,
                       double* v_ant, double* T_ant);
/* Asynchronous form of ixb_download_state, for writers that run beside the
 * next iterations (the restart and output files of main.f90:1327-1363 and
 * mod_postproceso.f90:225-365, which the reference writes from a blocking
 * `!$acc update self`).  On the handle's stream it snapshots the requested
 * arrays (a device-side copy in host layout) and returns; the copies to
 * the host run on a stream of their own, so the next ixb_step can start
 * at once.  The host arrays must stay valid, and should be pinned
 * (ixb_host_alloc) for the copies to overlap, until ixb_download_wait
 * returns.  A second asynchronous download waits on the device for the
 * first one's copies before reusing the snapshot. */
int ixb_download_state_async(ixb_handle* h, double* u, double* v, double* p, double* T, double* u_ant,
                             double* v_ant, double* T_ant);
/* Block until the last ixb_download_state_async of the handle has landed in
 * host memory.  It touches only that download's completion event, so a
 * writer thread may call it while the handle runs other calls, as long as
 * no new ixb_download_state_async starts meanwhile. */
int ixb_download_wait(ixb_handle* h);
/* Page-locked host memory for the asynchronous downloads (cudaMallocHost);
 * no counterpart in the reference. */
int ixb_host_alloc(size_t bytes, void** out);
int ixb_host_free(void* p);
/* Work arrays after the last iteration: au, av, b_o, Resu, corr_pres. */
int ixb_download_aux(ixb_handle* h, double* au, double* av, double* b_o, double* resu, double* corr_pres);

/* ---- the hot path ---- */
/* Exactly n passes of the ALGORITMO_SIMPLE body (main.f90:404-1200) with
 * the reference's inner loops, without the outer exit test. */
int ixb_simple_iterations(ixb_handle* h, int n, ixb_report* rep);
/* The ALGORITMO_SIMPLE loop of one time step, with the reference's exit
 * logic (main.f90:1202-1215). */
int ixb_simple_loop(ixb_handle* h, ixb_report* rep);
/* Nusselt monitor of ixb_simple_converge: the wall-averaged Nusselt number
 * of ixb_nusselt_y (vertical = 0: walls jj = 1 and nj+1, panels
 * ii = k0..k1 step 2) or ixb_nusselt_x (vertical = 1: walls ii = 1 and
 * mi+1, panels jj = k0..k1 step 2), evaluated every `every` outer
 * iterations on the device.  `wall` picks the monitored one (0: index 1,
 * 1: the last index). */
typedef struct {
  int vertical, k0, k1, wall;
  int every;            /* outer iterations between evaluations (>= 1) */
  int reserved;
  int64_t max_iters;    /* stop once this many outer iterations ran (checked every `every`) */
  double tol_dnu;       /* stop when |Nu - Nu of the previous evaluation| < tol_dnu */
  double tol_maxbo;     /* stop when maxbo < tol_maxbo (0: never) */
} ixb_nu_monitor;
/* Outer SIMPLE iterations (ixb_simple_iterations' passes, no outer exit
 * test) until the monitored Nusselt number settles: one CUDA graph launch,
 * the Nusselt numbers and the stopping test run on the device between
 * blocks of `every` iterations, with no host round trip.  Derived from the
 * reference's periodic Nusselt evaluation (main.f90:1226-1247,
 * nusselt_promedio_y of mod_postproceso.f90:100-215), which runs on the
 * host every 1000 time steps and stops nothing.  nu[2] (may be NULL): both
 * walls' Nusselt numbers at the last evaluation; dnu (may be NULL): the
 * monitored wall's last change (infinite after a single evaluation).
 * rep->exit_code: 3 |dNu| < tol_dnu, 4 maxbo < tol_maxbo, 5 max_iters. */
int ixb_simple_converge(ixb_handle* h, const ixb_nu_monitor* mon, ixb_report* rep, double* nu, double* dnu);
/* Time-step roll T_ant,u_ant,v_ant <- T,u,v (main.f90:1251-1270). */
int ixb_roll(ixb_handle* h);
/* One time step: ixb_simple_loop then ixb_roll (main.f90:391-1271 body). */
int ixb_step(ixb_handle* h, ixb_report* rep);
/* One phase of the iteration, for per-kernel checks: 0 u-y sweep, 1 u-x,
 * 2 v-y, 3 v-x, 4 p'-y, 5 p'-x, 6 p/u/v correction, 7 T-y, 8 T-x,
 * 9 u residual.  Phase 4 reads p' from the current corr_pres. */
int ixb_phase(ixb_handle* h, int which);
/* Device time of each phase 0..9 of ixb_phase: each phase is launched
 * `reps` times on the handle's stream, every launch bracketed by two CUDA
 * events; when flush_bytes > 0 a scratch buffer of that size is written
 * before every launch so the kernel starts with a cold L2.  ms[k] receives
 * the mean milliseconds per launch of phase k.  The state is advanced by the
 * launches (use on a scratch copy).  No reference counterpart: it measures
 * the kernels that replace the OpenACC regions. */
int ixb_time_phases(ixb_handle* h, int reps, size_t flush_bytes, double* ms);
/* Launch shape of one sweep (0..7 = u-y, u-x, v-y, v-x, p'-y, p'-x, T-y,
 * T-x): lines per CTA and threads per line, one of (1,128) (1,256) (1,512)
 * (2,64) (2,128) (4,32) (4,64) (4,128) (5,64) (5,128) (6,64) (6,128)
 * (8,32) (8,64) (8,128) (16,16) (16,32); each thread eliminates a chunk of
 * max(3, ceil(n/threads_per_line)) rows.  lines_per_cta = 0 restores the
 * default: x-lines one per CTA, 256 threads above 384 rows, else 128;
 * y-lines the fewest of 4, 5, 6 or 8 adjacent lines per CTA that keeps one
 * CTA per SM (8 beyond that), 128 threads per line from 160 rows, else 64.
 * No reference counterpart: the reference runs one sequential tridiagonal
 * per OpenACC gang. */
int ixb_set_sweep_shape(ixb_handle* h, int sweep, int lines_per_cta, int threads_per_line);
/* Kernels one outer iteration launches with the current launch shapes (one
 * inner pass per loop): one per sweep whose shape runs assembly and line
 * solve as one kernel (x-sweeps with one line per CTA; y-sweeps with 4 to
 * 16 lines per CTA), two per other sweep, plus the p/u/v correction and the
 * u residual, and the p' reset when the loop is host-driven
 * (IXB_NO_GRAPH=1) or IXB_DOWHILE=0.  IXB_SPLIT=1 in the environment keeps
 * every sweep at two kernels. */
int ixb_iteration_launches(ixb_handle* h, int* launches);
/* Autotuner for the launch shapes: for every sweep, times each candidate
 * shape `reps` times on the current state (a scratch buffer of flush_bytes
 * is written before every timed launch when flush_bytes > 0) and keeps the
 * fastest.  The state is restored afterwards.  chosen[2k], chosen[2k+1]
 * receive sweep k's lines per CTA and threads per line; ms[k] its mean
 * milliseconds per launch (either may be NULL). */
int ixb_autotune(ixb_handle* h, int reps, size_t flush_bytes, int* chosen, double* ms);
/* Overwrite corr_pres / au / av on the device (host arrays), for ixb_phase checks. */
int ixb_set_work(ixb_handle* h, const double* corr_pres, const double* au, const double* av);

/* ---- post-processing on the device ---- */
/* nusselt_promedio_y (source/mod_postproceso.f90:100-215): walls jj=1 and
 * jj=nj+1, integrated over ii = i0..i1 step 2. */
int ixb_nusselt_y(ixb_handle* h, int i0, int i1, double* nu0, double* nu1);
/* The same rule on the vertical walls ii=1 and ii=mi+1, over jj = j0..j1
 * step 2 (no counterpart in the reference; it only has the horizontal form). */
int ixb_nusselt_x(ixb_handle* h, int j0, int j1, double* nu0, double* nu1);

/* ---- batched line solver: tridiagonal (source/mod_solucionador.f90:25-47)
 * over many systems, DEVICE pointers.  Row i of system s is
 * a[i]x[i-1] + b[i]x[i] + c[i]x[i+1] = d[i]; a[0] and c[n-1] are ignored.
 * layout 0: system s row i at s*n + i (contiguous, x-lines);
 * layout 1: at i*nsys + s (interleaved, y-lines).
 * x may alias d.  a, b, c, d are not modified (unless x aliases d). ---- */
int ixb_tridiag_f64(const double* a, const double* b, const double* c, const double* d, double* x, int n,
                    int nsys, int layout, int solver, void* stream);
int ixb_tridiag_f32(const float* a, const float* b, const float* c, const float* d, float* x, int n,
                    int nsys, int layout, int solver, void* stream);
/* The hybrid solves above run their copies through the tensor/bulk-copy
 * engine and wait on them for a bounded time; a wait that expires leaves the
 * affected systems unwritten and is recorded on the device.  This call waits
 * for all work on the current device, then returns IXB_ETIMEOUT if such a
 * wait expired since the previous call (and clears the record), IXB_ECUDA if
 * the device reports an error, else IXB_OK.  No counterpart in the
 * reference, whose solver has no waits. */
int ixb_tridiag_status(void);
/* Failure-detection hook, no counterpart in the reference: the number of
 * polls the first copy wait of every CTA of the streamed contiguous solve
 * (hybrid solver, layout 0) may take before it counts as expired; polls < 0
 * restores the default (2^22 polls, at most about two seconds).  With 0 the
 * first wait expires at once: each CTA records the timeout, waits at the
 * default bound for its copies already in flight, and returns without
 * writing, so ixb_tridiag_status reports IXB_ETIMEOUT and the device stays
 * usable.  Process-wide; for tests only. */
int ixb_tridiag_set_first_wait_limit(int polls);

/* Allocation-free form of ixb_tridiag_f64 (no counterpart in the reference),
 * for callers that cannot let a library allocate device memory during their
 * run: e.g. a driver whose GPU memory is owned by its OpenACC runtime or by a
 * pool reserved at start-up, a solver sharing a GPU under a fixed memory
 * budget, or a loop that must avoid the implicit synchronisation an
 * allocation can cause.  Same arguments and results as ixb_tridiag_f64; it
 * calls no cudaMalloc/cudaFree or other allocating routine.
 * - layout 0 needs no scratch (systems are staged in shared memory).
 * - layout 1 keeps its scratch in a fixed 8 MiB array that belongs to the
 *   library's device image (one per GPU that loads the library, held until
 *   the process exits): n*nsys must not exceed IXB_NOALLOC_MAX_ELEMS, larger
 *   calls return IXB_EINVAL without launching anything.
 * - A layout-1 call outside stream capture looks up the array's device
 *   address (cudaGetSymbolAddress) with that device current, so a context
 *   re-created after cudaDeviceReset is picked up; a call on a capturing
 *   stream reuses the address of the last uncaptured call on that device.
 *   Make a first uncaptured layout-1 call on a device before capturing one
 *   (otherwise the captured call returns IXB_ECUDA).
 * - Every call shares the one array; nothing in it needs to start at zero
 *   (each element is written before it is read), but calls whose kernels
 *   overlap on the GPU (different streams, or different host threads) race
 *   on it: serialise them. */
#define IXB_NOALLOC_MAX_ELEMS (1 << 20)
int ixb_tridiag_f64_noalloc(const double* a, const double* b, const double* c, const double* d, double* x, int n,
                            int nsys, int layout, int solver, void* stream);

/* ---- energy equation with the flow held fixed, and its discrete adjoint ----
 * No counterpart in the reference.  ixb_energy_iterations runs n passes of
 * the two T sweeps (T-y then T-x, main.f90:985-1136) at the current u, v.
 * ixb_adjoint_energy returns, for the same K passes from the current state,
 * the gradient of the hot-wall Nusselt number nu0 of ixb_nusselt_x(h, j0, j1)
 * with respect to the boundary value of every T x-line on side a (x = 0):
 * grad[jj-1] = d nu0 / d value(jj), jj = 1..nj+1 (zero where the line is not
 * solved).  The map is affine in T with u, v fixed, so the gradient is exact
 * (transposed line solves, no stored forward states); the state is left
 * unchanged; IXB_ETIMEOUT if a transposed line solve's copies did not arrive
 * within their bounded wait.  ixb_set_bc_values sets the per-line values of one side of a
 * boundary table (a per-node profile, beyond the reference's 15 segments),
 * keeping each line's type. */
/* ---- discrete adjoint of the full coupled SIMPLE iteration ----
 * No counterpart in the reference.  K outer iterations from the current state,
 * each one pass of every equation (u-y, u-x, v-y, v-x, p'-y from p' = 0,
 * p'-x, the velocity/pressure update, T-y, T-x: main.f90:404-1136 with
 * iter_ecuaci_max = 0), then nu0 = the hot-wall Nusselt number of
 * ixb_nusselt_x(h, j0, j1).  With grad (nj+1 entries, may be NULL for the
 * forward only): d nu0 / d value of the side-a T boundary row of every
 * x-line jj (grad[jj-1]; lines 1 and nj+1 are not solved and get 0),
 * through the momentum, pressure-correction and energy sweeps and their
 * coupling (buoyancy, convection): the adjoint for flows that depend on T.
 * The forward state is saved every C iterations; each segment is recomputed
 * storing the state after every phase (16 fields per iteration, so device
 * memory grows with C) and reversed with transposed line solves.  Leaves
 * the state of the K-iteration forward run.  Binary64 handles only
 * (IXB_EINVAL otherwise). */
int ixb_adjoint_simple(ixb_handle* h, int K, int C, int j0, int j1, double* grad, double* nu0);
int ixb_energy_iterations(ixb_handle* h, int n);
int ixb_adjoint_energy(ixb_handle* h, int K, int j0, int j1, double* grad);
int ixb_set_bc_values(ixb_handle* h, int var, int side, const double* values);
/* The same gradient through K outer SIMPLE iterations (ixb_simple_iterations
 * from the current state) whose flow evolves but does not depend on the
 * temperature: Ri = Riy = 0 (forced convection), else IXB_EINVAL.  Then T
 * after K iterations is a composition of affine T passes, those of iteration
 * k with the coefficients of that iteration's velocities, and the gradient is
 * exact.  The call runs the K iterations, checkpointing the seven state
 * fields every C iterations (device memory for K/C + 1 checkpoints and C
 * velocity pairs), then reverses them segment by segment, recomputing each
 * segment from its checkpoint; it leaves the state after the K iterations
 * and, if nu0 is not NULL, stores nu0 of ixb_nusselt_x(h, j0, j1) there.
 * Binary64 form (IXB_PREC_FP64) for the exact gradient. */
int ixb_adjoint_energy_coupled(ixb_handle* h, int K, int C, int j0, int j1, double* grad, double* nu0);

/* ---- batched cavities: many instances, one launch per phase ----
 * No counterpart in the reference, which runs one case per process.  A
 * batch owns `count` instances of sizes mi[i] x nj[i] (4..1024 each), all in
 * the same precision mode.  Each instance is an ordinary handle: set its
 * mesh, parameters, boundary tables, sources and state, and read its state
 * and Nusselt numbers, through the single-instance calls on the handle
 * ixb_batch_instance returns (the batch owns it: do not destroy it).  One
 * outer iteration of the batch runs every phase of the SIMPLE iteration as
 * one launch over the work of all active instances, with one pass of each
 * equation (the reference's loops with iter_ecuaci_max = 0); the loop is a
 * single CUDA graph.  An instance stops when its outer test (main.f90:1202:
 * maxbo < conv_paso and residuo < conv_resi) holds or a norm is not finite. */
typedef struct ixb_batch ixb_batch;
int ixb_batch_create(int count, const int* mi, const int* nj, int prec_mode, ixb_batch** out);
int ixb_batch_destroy(ixb_batch* b);
int ixb_batch_instance(ixb_batch* b, int i, ixb_handle** h);
/* Launch shape of sweep `sweep` (IXB_SWEEP_* order) for every instance, as
 * ixb_set_sweep_shape; 0, 0 restores the default. */
int ixb_batch_set_sweep_shape(ixb_batch* b, int sweep, int lines_per_cta, int threads_per_line);
/* Time the seven launch shapes of every sweep on the batch (reps batched
 * iterations each) and keep the fastest; chosen[2*s], chosen[2*s+1] and
 * ms[s] (may be null) receive the choice and its time per sweep.  The state
 * of every instance is saved before and restored after. */
int ixb_batch_autotune(ixb_batch* b, int reps, int* chosen, double* ms);
/* Mark every instance active again with its counters cleared. */
int ixb_batch_restart(ixb_batch* b);
/* Run up to max_iters outer iterations of the active instances; *n_active
 * receives how many are still active afterwards. */
int ixb_batch_iterate(ixb_batch* b, int max_iters, int* n_active);
/* Instance i after the last ixb_batch_iterate: norms, iterations done since
 * the last restart (n_simple), exit_code 0 running, 1 converged, 2 stopped
 * by the iteration budget, 3 non-finite norm (status IXB_ENONFINITE). */
int ixb_batch_report(ixb_batch* b, int i, ixb_report* out);

/* ---- mesh generation and mesh/state files (host only, no GPU needed) ---- */
#define IXB_MESH_UNIF 0 /* malla/malla_irr.f90:97-100 */
#define IXB_MESH_TUBO 1 /* erf clustering at both walls, malla_irr.f90:81-89 */
#define IXB_MESH_CENT 2 /* sinh clustering around `centre` (tau = param), malla_irr.f90:54-64 */
#define IXB_MESH_TANH 3 /* two-sided tanh wall clustering, parameter = stretching; no counterpart
                           in malla_irr.f90 */
/* n u- (or v-) node coordinates of one axis on [0, length]. */
int ixb_mesh_axis(int kind, int n, double length, double param, double centre, double* nodes);
/* Staggered mesh of malla_irr.f90: xu (mi), yv (nj) from ixb_mesh_axis (the
 * cent kind centred on the middle of the axis), p nodes xp (mi+1), yp (nj+1)
 * at the midpoints plus one node half a cell outside each wall (:66-77,
 * :101-106); every coordinate rounded to 15 significant digits, as the
 * D23.15 mesh files hold them. */
int ixb_staggered_mesh(int mi, int nj, int xkind, double xparam, int ykind, double yparam, double ao, double bo,
                       double* xu, double* yv, double* xp, double* yp);
/* The three mesh/state files (written by malla_irr.f90:176-203, read by
 * lectura_mallas_escalonadas, source/mod_malla.f90:137-162): header
 * "i_0 i_1 iter a", then per node (DO jj, DO ii) "x y u" (u file), "x y v"
 * (v file), "x y T p" (p file) in D23.15.  Arrays in the Fortran shapes
 * u(mi,nj+1), v(mi+1,nj), T/p(mi+1,nj+1), column-major.  Returns IXB_EIO when a
 * file cannot be opened, written or parsed. */
int ixb_write_state_files(const char* ufile, const char* vfile, const char* pfile, int mi, int nj, const double* xu,
                          const double* yv, const double* xp, const double* yp, const double* u, const double* v,
                          const double* T, const double* p, int i0, int i1, int iter, double a);
int ixb_read_state_files(const char* ufile, const char* vfile, const char* pfile, int mi, int nj, double* xu,
                         double* yv, double* xp, double* yp, double* u, double* v, double* T, double* p, int* i0,
                         int* i1, int* iter, double* a);

/* ---- immersed solid bodies (host only, no GPU needed) ---- */
#define IXB_BODY_BOX 0    /* prm = {x0, x1, y0, y1}: x0 <= x <= x1, y0 <= y <= y1 */
#define IXB_BODY_REGION 1 /* prm = {y0, y1, s0, c0, s1, c1}: y0 <= y <= y1, s0*y + c0 <= x <= s1*y + c1
                             (en_region_tipo1, source/mod_front_inmersa.f90:188-207) */
#define IXB_BODY_TRIAN 2  /* definir_cuerpo 'trian' (mod_front_inmersa.f90:73-99): u, v */
#define IXB_BODY_CUADR 3  /* definir_cuerpo 'cuadr' (:101-133): u, v */
#define IXB_BODY_CHIME 4  /* definir_cuerpo 'chime' (:135-177): u, v, and T held at 1 */
#define IXB_BODY_VEL 1    /* flags: penalty sources on u and v (held at 1e40 / 1e51 = 1e-11 in the body) */
#define IXB_BODY_TEMP 2   /* flags: T held at t_value in the body */
/* Penalty sources of an immersed body (definir_cuerpo, mod_front_inmersa.f90:
 * 54-179), for ixb_set_sources: every p node (xp(ii), yp(jj)) inside the body
 * sets fuente_lin = -1e51 and fuente_con = 1e40 (u, v) or 1e51 * t_value (T)
 * at (ii, jj) of the u (mi, nj+1), v (mi+1, nj) and T (mi+1, nj+1) arrays,
 * column-major; other entries are left as they are, so bodies accumulate.
 * The reference also writes u at ii = mi+1 and v at jj = nj+1, past the ends
 * of those arrays; those writes are dropped.  For the three fixed shapes prm,
 * flags and t_value are ignored.  Arrays of variables the body does not touch
 * may be NULL. */
int ixb_body_sources(int mi, int nj, const double* xp, const double* yp, int shape, const double* prm, int flags,
                     double t_value, double* fcon_u, double* flin_u, double* fcon_v, double* flin_v, double* fcon_t,
                     double* flin_t);

/* ---- host-side inputs (no GPU needed) ---- */
/* lectura_cond_frontera index rule (source/mod_cond_frontera.f90:114-238):
 * for side 0/2 ('a'/'c') the divisions are located on `yy` (nn entries), for
 * 1/3 ('b'/'d') on `xx` (mm entries). */
int ixb_bc_locate(int side, int ndivis, const double* x1, const int* type, const double* value,
                  const double* xx, int mm, const double* yy, int nn, ixb_bc_side* out);
/* Read cond_frontera{u,v,t}.dat: four sides, each "variable side ndivis"
 * followed by ndivis lines "x0 x1 type value". */
int ixb_read_bc_file(const char* path, const double* xx, int mm, const double* yy, int nn,
                     ixb_bc_side out[4]);

#ifdef __cplusplus
}
#endif
#endif /* IXB_H */
