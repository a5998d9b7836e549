// ixb_internal.h -- host-side declarations shared by the library's
// translation units (not part of the public ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#include "../../include/ixb.h"
#include "ixb_device.cuh"

namespace ixb {

// With IXB_PDL=1 in the environment the kernels of the SIMPLE loop are
// launched with programmatic stream serialisation: each one may be placed on
// the GPU while its predecessor finishes and waits for the predecessor's
// completion (and memory) at entry (IXB_PDL_ENTRY), so results are
// unchanged.  Off by default: at 701x301 it measured 115.9 us per outer
// iteration against 109.9 us without it (refined; binary64 138 against
// 120 us).
bool pdl_enabled();
// fused sweeps set a shared-memory carveout of one wave of CTAs unless IXB_CARVEOUT=0
bool carveout_enabled();
// fused sweeps (one kernel per sweep) unless IXB_SPLIT=1
bool fused_enabled();
template <class... KArgs, class... Args>
inline cudaError_t launch_k(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                            Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

enum NormId { N_DV = 0, N_DP, N_BO, N_DT, N_RES, N_COUNT };

// Loop control carried by a kernel of the graph-driven SIMPLE loop (ctl
// null: none, as in the host-driven loop): the kernel that finishes a norm
// applies the exit test that reads it and sets the loop's conditional node
// (ixb_ctl.cuh).
struct Ctl;
struct CtlRef {
  Ctl* ctl;
  const double* norms;
  cudaGraphConditionalHandle cond;   // the loop this kernel ends or opens
  cudaGraphConditionalHandle cond2;  // outer step: the momentum loop to reopen
  int which;                         // inner step: 0 momentum, 1 pressure, 2 energy
};

// Line-solve forms of the sweep kernels: IXB_SOLVER_HYBRID (0) and
// IXB_SOLVER_EXACT (1) of the public ABI, plus the mixed-precision form a
// handle created with IXB_PREC_FP32_REFINED runs in place of the hybrid one.
constexpr int SOLVER_MIXED = 2;

template <int EQ>
struct EqIsX { static constexpr bool value = (EQ & 1) != 0; };

// Arithmetic types of one sweep.  The binary64 solvers use binary64
// throughout.  The mixed solver (handle precision IXB_PREC_FP32_REFINED)
// assembles every row in binary64 and stages and solves the lines in
// binary32, each row scaled to a unit diagonal first (so that immersed-body
// penalties of ~1e51, or the vanishing p' coefficients inside a body, stay
// representable).  The u, v and T rows are a defect correction (DC): the
// binary64 residual d - A x of the current values is solved for in binary32
// and the correction added back in binary64, so the fixed point of these
// equations is the binary64 one.  The p' rows are solved outright in
// binary32 (p' only steers the iteration; it vanishes at convergence), around
// a binary64 mass source b_o.
template <int SOLVER, int EQ>
struct SweepTypes {
  static constexpr bool MIX = SOLVER == SOLVER_MIXED;
  static constexpr bool DC = MIX && EQ != EQ_PY && EQ != EQ_PX;
  using S = typename std::conditional<MIX, float, double>::type;  // staged rows, line solve
};

// x-sweep tiles: 64 consecutive rows of 8 lines; y-sweep tiles: 32 lines
// (adjacent ii) x 16 rows, written back through shared memory as 16-row
// runs of each line.  Each of the 256 threads assembles kAsmCPT cells.
constexpr int kAsmThreads = 256;
constexpr int kAsmCPT = 2;  // cells per thread (their loads in flight together)
constexpr int kAsmXR = 64, kAsmXL = 4 * kAsmCPT;
constexpr int kAsmYL = 32, kAsmYR = 8 * kAsmCPT;

__host__ __device__ constexpr int asm_tiles(bool x, int n, int nlines) {
  return x ? ((n + kAsmXR - 1) / kAsmXR) * ((nlines + kAsmXL - 1) / kAsmXL)
           : ((nlines + kAsmYL - 1) / kAsmYL) * ((n + kAsmYR - 1) / kAsmYR);
}

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

// One instance of a batched launch (see ixb_batch.cu): its views, and its
// work items first .. first+count-1 in the launch's item list.
template <class S>
struct AsmInst {
  Geo<double> G;
  SweepIO<double> io;
  Coef<S> co;
  int n, line_lo, line_hi;
  int first, count;
};

// per-equation assembly launchers (ixb_sweep_<eq>.cu: exact,
// ixb_sweep_<eq>_fast.cu: hybrid, ixb_sweep_<eq>_mixed.cu: mixed precision)
template <int EQ, int SOLVER>
cudaError_t assemble_launch(const SweepShape& s, const Geo<double>& G, const SweepIO<double>& io,
                            const StageBuf& buf, cudaStream_t st);
template <int EQ, int SOLVER>
cudaError_t assemble_batch_launch(const void* inst, const int2* items, int nitems, const int* active,
                                  const BatchNorm& bn, cudaStream_t st);

// line solve of a sweep (ixb_solve.cu): staged rows in, field out
// The u residual (residuo_u, mod_ec_momento.f90:1107-1266, main.f90:1169-1199)
// of the rows a fused T-x sweep has just solved, its norm, and the outer
// test after the energy loop's last pass (graph only; resu null: off).  The
// residual of u-row jj reads T on row jj only, which is that sweep's line jj.
struct ResidIO {
  const double *u, *v, *p, *u_ant, *fcon, *flin;
  double* resu;
  NormSlot ns;
  CtlRef outer;
};

struct SolveIO {
  const void* coef;     // a | b | c | d, `stride` elements each
  size_t stride;
  int P;
  const double* in;     // swept field, current values (copied on unsolved lines)
  double* out;          // swept field, new values
  const double* prev;   // field at the start of the inner pass (null: zero)
  NormSlot nrm0;        // ||out - prev|| over interior rows of solved lines
  CtlRef ctl;           // inner-loop test after nrm0 (graph only)
  int LD;
  int m, mp;            // chunk rows per thread, padded pitch
  ResidIO res;          // fused T-x sweeps only
};
// Launch shapes of the line sweeps (lines per CTA, threads per line); every
// sweep runs in one of them (ixb_set_sweep_shape, the autotuners).  The
// line-solve kernels are instantiated for each (IXB_SWEEP_SHAPES, ixb_solve.cu).
// 5 and 6 lines per CTA put a 701-line y-sweep on 141 or 117 CTAs (one per
// SM) where 8 lines leave 60 of the 148 SMs idle.
constexpr int kNumShapes = 17;
constexpr int kShapeList[kNumShapes][2] = {{1, 128}, {1, 256}, {1, 512}, {2, 64},  {2, 128}, {4, 32},
                                          {4, 64},  {4, 128}, {5, 64},  {5, 128}, {6, 64},  {6, 128},
                                          {8, 32},  {8, 64},  {8, 128}, {16, 16}, {16, 32}};

// Launch shapes (lines per CTA, threads per line) of the fused sweeps:
// x-sweeps one line per CTA; y-sweeps 4 to 16 adjacent lines per CTA, so
// that a warp's field reads span adjacent lines (with 2 lines a warp reads
// 16 separate 16-byte pieces and the fused y-sweep measured twice as slow
// as its two kernels).
#define IXB_FUSED_X_SHAPES(X_) X_(1, 128) X_(1, 256) X_(1, 512)
#define IXB_FUSED_Y_SHAPES(X_) \
  X_(4, 32) X_(4, 64) X_(4, 128) X_(5, 64) X_(5, 128) X_(6, 64) X_(6, 128) X_(8, 32) X_(8, 64) X_(8, 128) \
  X_(16, 16) X_(16, 32)
inline bool fused_shape(int eq, int tl, int g) {
  bool hit = false;
#define IXB_HIT_(TL_, G_) hit = hit || (tl == TL_ && g == G_);
  if (eq & 1) { IXB_FUSED_X_SHAPES(IXB_HIT_) }  // x-sweeps are the odd ones (EqIsX)
  else { IXB_FUSED_Y_SHAPES(IXB_HIT_) }
#undef IXB_HIT_
  return hit;
}
// fused sweep (assembly into the solve's shared memory, one launch;
// ixb_sweep.cuh); cudaErrorNotSupported for shapes it does not cover
template <int EQ, int SOLVER>
cudaError_t fused_launch(const SweepShape& s, const Geo<double>& G, const SweepIO<double>& io, const SolveIO& so,
                           cudaStream_t st);
// one instance of a batched line solve
struct SolveInst {
  SolveIO io;
  int n, line_lo, line_hi, nfull;
  int first, count;  // its work items in the launch's item list
};
// one instance of a batched fused sweep: its assembly view and its line solve
struct FusedInst {
  Geo<double> G;
  SweepIO<double> io;
  SolveInst s;
};
template <int EQ, int SOLVER>
cudaError_t fused_batch_launch(int tl, int g, size_t smem, const FusedInst* inst, const int2* items, int nitems,
                               const int* active, const BatchNorm& bn_asm, const BatchNorm& bn_sol,
                               cudaStream_t st);
// form: IXB_SOLVER_HYBRID, IXB_SOLVER_EXACT or SOLVER_MIXED; x: line along
// ii; dc: the staged right-hand sides are binary64 residuals whose solution
// is added to `in`
cudaError_t solve_launch(int form, bool x, bool dc, const SweepShape& s, const SolveIO& io, cudaStream_t st);
int solve_blocks_per_sm(int form, bool x, bool dc, const SweepShape& s);
cudaError_t solve_set_smem_limits(int bytes);
// batched line solve with one launch shape (TL lines x G threads) for all
// instances; smem: shared memory of the largest instance's lines
cudaError_t solve_batch_launch(int form, bool x, bool dc, int tl, int g, size_t smem, const SolveInst* inst,
                               const int2* items, int nitems, const int* active, const BatchNorm& bn,
                               cudaStream_t st);
int sweep_occupancy(int eq, int solver, const SweepShape& s);
int max_sweep_lines(int mi, int nj);

// one instance of a batched correction / residual launch; work items are
// blocks of kCellChunk cells
constexpr int kCellChunk = 256;
struct CellInst {
  Geo<double> G;
  double *u, *v, *p, *resu;
  const double *pc, *au, *av, *T, *u_ant, *fcon, *flin;
  int first, count;  // its residual work items in the launch's item list
};
cudaError_t correct_batch_launch(const CellInst* inst, const int2* items, int nitems, const int* active, int fast,
                                 cudaStream_t st);
cudaError_t residual_batch_launch(const CellInst* inst, const int2* items, int nitems, const int* active,
                                  const BatchNorm& bn, int fast, cudaStream_t st);

// kernel launchers (ixb_kernels.cu); return cudaError_t
// rio (T-x in a fused shape only): the u residual rides on the sweep
cudaError_t launch_sweep_f64(int eq, int solver, const SweepShape& s, const Geo<double>& G,
                             const SweepIO<double>& io, const StageBuf& buf, cudaStream_t st,
                             const CtlRef& ctl = CtlRef{}, const ResidIO* rio = nullptr);
cudaError_t launch_correct_f64(const Geo<double>& G, double* u, double* v, double* p, const double* pc,
                               const double* au, const double* av, int fast, cudaStream_t st,
                               const CtlRef& gate = CtlRef{});
cudaError_t launch_residual_f64(const Geo<double>& G, const double* u, const double* v, const double* T,
                                const double* p, const double* u_ant, const double* fcon, const double* flin,
                                double* resu, NormSlot ns, int fast, cudaStream_t st,
                                const CtlRef& outer = CtlRef{});
// p' = 0 over a whole field, opening the pressure loop (graph only)
cudaError_t launch_preset_f64(double* pc, size_t n, const CtlRef& gate, cudaStream_t st);
int residual_grid(int mi, int nj);
// Nusselt numbers of both walls (out2); with `mon` set, the wall and panel
// range come from the monitor fields of `mon`, and the monitor's stopping
// test sets `cond` (graph only)
cudaError_t launch_nusselt_f64(const Geo<double>& G, const double* T, const double* xp, const double* yp,
                               int vertical, int k0, int k1, double* out2, cudaStream_t st, Ctl* mon = nullptr,
                               cudaGraphConditionalHandle cond = 0);
cudaError_t sweep_set_smem_limits();
cudaError_t launch_tables_f64(const Geo<double>& G, double* met, double* tab, cudaStream_t st);

// batched standalone tridiagonal solvers (ixb_tridiag.cu)
cudaError_t tridiag_f64(const double* a, const double* b, const double* c, const double* d, double* x, int n,
                        int nsys, int layout, int solver, cudaStream_t st);
cudaError_t tridiag_f32(const float* a, const float* b, const float* c, const float* d, float* x, int n,
                        int nsys, int layout, int solver, cudaStream_t st);
// reads and clears the flag set when a line-solve kernel's bounded wait on
// its copies expired (synchronous)
cudaError_t tridiag_take_timeout(int* flag);

}  // namespace ixb
