// ixb_internal.h -- host-side declarations shared by the library's
// translation units (not part of the public ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ixb.h"
#include "ixb_device.cuh"

namespace ixb {

enum NormId { N_DV = 0, N_DP, N_BO, N_DT, N_RES, N_COUNT };

// Line-solve forms of the sweep kernels: IXB_SOLVER_HYBRID (0) and
// IXB_SOLVER_EXACT (1) of the public ABI, plus the mixed-precision form a
// handle created with IXB_PREC_FP32_REFINED runs in place of the hybrid one.
constexpr int SOLVER_MIXED = 2;

// launch shape of one sweep
struct SweepShape {
  int n;          // rows per line
  int line_lo;    // first solved line (1-based)
  int line_hi;    // last solved line
  int nfull;      // lines of the field (unsolved ones are copied)
  int tl;         // lines per CTA
  int g;          // threads per line
  int nt;         // threads per CTA (tl * g)
  int m, mp;      // chunk rows per thread, padded pitch
  int rs;         // reduced-system solver (RS_PCR / RS_WARP)
  size_t smem;    // dynamic shared memory bytes
  int grid;       // CTAs
};

// Shape of sweep `eq` with tl lines per CTA and g threads per line
// (tl * g = 128 or 256; chunks of max(3, ceil(n/g)) rows).
SweepShape sweep_shape(int eq, int mi, int nj, int real_bytes, int tl, int g);

// Rows of one sweep staged between its assembly and its line solve: four
// arrays a | b | c | d of `stride` elements (binary64, or binary32 in the
// mixed form), line L of the sweep at (L - line_lo) * P.
template <class S>
struct Coef {
  S *a, *b, *c, *d;
  int P;
};
struct StageBuf {
  void* base;
  size_t stride;  // elements per array
  int P;          // row pitch of a line (>= rows per line, multiple of 32)
};

// Assembly grids are capped (grid-stride over tiles) so that the per-CTA
// partials of a norm fit the handle's partials buffer.
constexpr int kAsmGridCap = 148 * 8;

// per-equation assembly launchers (ixb_sweep_<eq>.cu: exact,
// ixb_sweep_<eq>_fast.cu: hybrid, ixb_sweep_<eq>_mixed.cu: mixed precision)
template <int EQ, int SOLVER>
cudaError_t assemble_launch(const SweepShape& s, const Geo<double>& Gd, const Geo<float>& Gf,
                            const SweepIO<double>& io, const StageBuf& buf, cudaStream_t st);

// line solve of a sweep (ixb_solve.cu): staged rows in, field out
struct SolveIO {
  const void* coef;     // a | b | c | d, `stride` elements each
  size_t stride;
  int P;
  const double* in;     // swept field, current values (copied on unsolved lines)
  double* out;          // swept field, new values
  const double* prev;   // field at the start of the inner pass (null: zero)
  NormSlot nrm0;        // ||out - prev|| over interior rows of solved lines
  int LD;
  int m, mp;            // chunk rows per thread, padded pitch
};
// form: IXB_SOLVER_HYBRID, IXB_SOLVER_EXACT or SOLVER_MIXED; x: line along
// ii; dc: the staged right-hand sides are binary64 residuals whose solution
// is added to `in`
cudaError_t solve_launch(int form, bool x, bool dc, const SweepShape& s, const SolveIO& io, cudaStream_t st);
int solve_blocks_per_sm(int form, bool x, bool dc, const SweepShape& s);
cudaError_t solve_set_smem_limits(int bytes);
int sweep_occupancy(int eq, int solver, const SweepShape& s);
int max_sweep_lines(int mi, int nj);

// kernel launchers (ixb_kernels.cu); return cudaError_t
cudaError_t launch_sweep_f64(int eq, int solver, const SweepShape& s, const Geo<double>& G,
                             const Geo<float>& Gf, const SweepIO<double>& io, const StageBuf& buf,
                             cudaStream_t st);
cudaError_t launch_correct_f64(const Geo<double>& G, double* u, double* v, double* p, const double* pc,
                               const double* au, const double* av, int fast, cudaStream_t st);
cudaError_t launch_residual_f64(const Geo<double>& G, const double* u, const double* v, const double* T,
                                const double* p, const double* u_ant, const double* fcon, const double* flin,
                                double* resu, NormSlot ns, int fast, cudaStream_t st);
int residual_grid(int mi, int nj);
cudaError_t launch_nusselt_f64(const Geo<double>& G, const double* T, const double* xp, const double* yp,
                               int vertical, int k0, int k1, double* out2, cudaStream_t st);
cudaError_t sweep_set_smem_limits();
cudaError_t launch_tables_f64(const Geo<double>& G, double* met, double* tab, cudaStream_t st);
cudaError_t launch_narrow_f32(const double* src, float* dst, size_t n, cudaStream_t st);

// batched standalone tridiagonal solvers (ixb_tridiag.cu)
cudaError_t tridiag_f64(const double* a, const double* b, const double* c, const double* d, double* x, int n,
                        int nsys, int layout, int solver, cudaStream_t st);
cudaError_t tridiag_f32(const float* a, const float* b, const float* c, const float* d, float* x, int n,
                        int nsys, int layout, int solver, cudaStream_t st);

}  // namespace ixb
