// ixb_tridiag.cu -- batched tridiagonal solves over device arrays, the
// batched form of tridiagonal (source/mod_solucionador.f90:25-47).
//
// layout 0 (each system contiguous, like the reference's x-lines): a CTA
// stages TL systems into shared memory with coalesced loads, G = 256/TL
// threads per system solve it (the chunked Thomas-PCR hybrid, or the exact
// sequential Thomas on one thread), and the solution is written back
// coalesced.
//
// layout 1 (systems interleaved, row i of system s at i*nsys+s, like the
// y-lines of a column-major field): the hybrid solver runs the cluster
// kernel below (tri_strided_kernel: groups of 128-byte row segments in 2-D
// tensor tiles, n <= 4096).  The exact solver, and sizes or alignments that
// kernel does not take, use one thread per system walking the rows;
// consecutive threads touch consecutive addresses.  Its forward sweep keeps
// the modified diagonal (exact) or normalised super-diagonal (hybrid) in a
// scratch array of n*nsys elements taken from the stream-ordered allocator,
// and the modified right-hand side in x.
#include <cooperative_groups.h>
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "ixb_internal.h"

namespace ixb {

template <class R, int SOLVER, int TL, int G>
__global__ void __launch_bounds__(TL * G) tri_contig_kernel(const R* __restrict__ a, const R* __restrict__ b,
                                                            const R* __restrict__ c, const R* __restrict__ d,
                                                            R* x, int n, int nsys, int m, int mp) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* sm = reinterpret_cast<R*>(smem_raw);
  const int npad = G * m;
  const size_t LS = line_smem_elems(G, mp), arr = (size_t)G * mp;
  const long long s0 = (long long)blockIdx.x * TL;
  for (int idx = threadIdx.x; idx < TL * npad; idx += TL * G) {
    const int l = idx / npad, r = idx - l * npad;
    const long long s = s0 + l;
    if (s >= nsys) continue;
    R ra = R(0), rb = R(1), rc = R(0), rd = R(0);
    if (r < n) {
      const size_t g = (size_t)s * n + r;
      ra = r == 0 ? R(0) : a[g];
      rb = b[g];
      rc = r == n - 1 ? R(0) : c[g];
      rd = d[g];
    }
    const int ch = r / m;
    const size_t o = (size_t)l * LS + (size_t)ch * mp + (r - ch * m);
    sm[o] = ra; sm[o + arr] = rb; sm[o + 2 * arr] = rc; sm[o + 3 * arr] = rd;
  }
  __syncthreads();
  {
    const int l = threadIdx.x / G;
    const bool active = s0 + l < nsys;
    R* line = sm + (size_t)l * LS;
    if (SOLVER == IXB_SOLVER_EXACT) {
      if (active && threadIdx.x % G == 0) thomas_exact(line, line + arr, line + 2 * arr, line + 3 * arr, n, m, mp);
    } else {
      chunk_solve<R, G>(line, m, mp, active, RS_WARP);
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < TL * n; idx += TL * G) {
    const int l = idx / n, r = idx - l * n;
    const long long s = s0 + l;
    if (s >= nsys) continue;
    const int ch = r / m;
    x[(size_t)s * n + r] = sm[(size_t)l * LS + 3 * arr + (size_t)ch * mp + (r - ch * m)];
  }
}

// One thread per interleaved system.  EXACT keeps the reference's operation
// order (modified diagonal in `work`); HYBRID uses the normalised Thomas form
// (c' in `work`).
template <class R, int SOLVER>
__global__ void __launch_bounds__(128) tri_inter_kernel(const R* __restrict__ a, const R* __restrict__ b,
                                                        const R* __restrict__ c, const R* __restrict__ d, R* x,
                                                        R* __restrict__ work, int n, int nsys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  const size_t S = (size_t)nsys;
  if (SOLVER == IXB_SOLVER_EXACT) {
    R bp = b[s], dp = d[s];
    work[s] = bp;
    x[s] = dp;
    for (int i = 1; i < n; ++i) {
      const size_t g = (size_t)i * S + s;
      const R q = a[g] / bp;
      dp = d[g] - q * dp;
      bp = b[g] - q * c[g - S];
      x[g] = dp;
      work[g] = bp;
    }
    R xn = dp / bp;
    x[(size_t)(n - 1) * S + s] = xn;
    for (int i = n - 2; i >= 0; --i) {
      const size_t g = (size_t)i * S + s;
      xn = (x[g] - c[g] * xn) / work[g];
      x[g] = xn;
    }
  } else {
    R r = R(1) / b[s];
    R cp = (n > 1 ? c[s] : R(0)) * r;
    R dp = d[s] * r;
    work[s] = cp;
    x[s] = dp;
    for (int i = 1; i < n; ++i) {
      const size_t g = (size_t)i * S + s;
      const R ai = a[g];
      r = R(1) / (b[g] - ai * cp);
      dp = (d[g] - ai * dp) * r;
      cp = (i < n - 1 ? c[g] : R(0)) * r;
      x[g] = dp;
      work[g] = cp;
    }
    R xn = dp;
    for (int i = n - 2; i >= 0; --i) {
      const size_t g = (size_t)i * S + s;
      xn = x[g] - work[g] * xn;
      x[g] = xn;
    }
  }
}

// ---------------------------------------------------------------------------
// Streamed contiguous solve (hybrid solver): a persistent CTA of 256 threads
// per SM slot walks its systems; while it solves system s from registers,
// the bulk-copy engine is already loading system s+grid into shared memory,
// and the solution leaves through a bulk shared->global copy.  Thread t owns
// rows t*M .. t*M+M-1 (M odd, so the 32 threads of a warp reading their own
// row j hit 32 different banks); it eliminates them in registers down to two
// rows (modified Thomas), the 512 reduced rows are solved by PCR in shared
// memory, and each thread back-substitutes its rows.  Every wait on the copy
// engine is bounded: on a timeout the CTA records it in g_tri_timeout, waits
// (bounded) for its copies still in flight and leaves without writing.
// ---------------------------------------------------------------------------
namespace {

constexpr int kStreamT = 256;       // threads per CTA (one system at a time)
constexpr int kSpinLimit = 1 << 22;  // bounded mbarrier polls (a hang guard)
__device__ int g_tri_timeout = 0;
// Poll limit of the streamed kernel's first wait of every CTA (its other
// waits, and the drain after a timeout, keep kSpinLimit); lowered only by
// ixb_tridiag_set_first_wait_limit, for failure-detection tests.
__device__ int g_tri_first_wait_polls = kSpinLimit;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void bulk_store(void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
               "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

__device__ __forceinline__ void bulk_store_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_store_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// At most `limit` polls, and no longer than about two seconds (%globaltimer).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int limit = kSpinLimit) {
  unsigned long long t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (int i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 255) {
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      if (t - t0 > 2000000000ull) return false;
    }
  }
  return false;
}

// Shared memory of the streamed kernel: 4 row arrays of NP = 256*M
// elements (the copy target), the solution buffer (NP), the PCR buffers
// (12*256) and the mbarrier.
template <class R, int M>
__host__ __device__ constexpr size_t stream_smem_bytes() {
  return ((size_t)5 * kStreamT * M + 12 * kStreamT) * sizeof(R) + 16;
}

template <class R, int M>
__global__ void __launch_bounds__(kStreamT, 1) tri_stream_kernel(const R* __restrict__ a, const R* __restrict__ b,
                                                                 const R* __restrict__ c, const R* __restrict__ d,
                                                                 R* __restrict__ x, int n, int nsys) {
  constexpr int NP = kStreamT * M;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* buf = reinterpret_cast<R*>(smem_raw);  // a | b | c | d, NP each
  R* xbuf = buf + 4 * NP;
  R* red = xbuf + NP;
  uint64_t* bar = reinterpret_cast<uint64_t*>(red + 12 * kStreamT);
  const int tid = threadIdx.x;
  const unsigned bytes = (unsigned)n * sizeof(R);
  // identity rows pad every system to NP rows; the copies never touch them
  for (int r = n + tid; r < NP; r += kStreamT) {
    buf[r] = R(0); buf[NP + r] = R(1); buf[2 * NP + r] = R(0); buf[3 * NP + r] = R(0);
  }
  if (tid == 0) mbar_init(bar);
  __syncthreads();
  auto issue = [&](int s) {
    const size_t off = (size_t)s * n;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier reads of buf precede the copies
    mbar_expect_tx(bar, 4 * bytes);
    bulk_load(buf, a + off, bytes, bar);
    bulk_load(buf + NP, b + off, bytes, bar);
    bulk_load(buf + 2 * NP, c + off, bytes, bar);
    bulk_load(buf + 3 * NP, d + off, bytes, bar);
  };
  if (tid == 0 && blockIdx.x < nsys) issue(blockIdx.x);
  const int first_limit = *(volatile int*)&g_tri_first_wait_polls;
  unsigned parity = 0;
  bool failed = false;
  for (int s = blockIdx.x; s < nsys; s += gridDim.x) {
    const bool ok = mbar_wait_bounded(bar, parity, s == (int)blockIdx.x ? first_limit : kSpinLimit);
    if (__syncthreads_or(!ok)) { failed = true; break; }
    parity ^= 1;
    // own rows into registers (row 0 has no a, row n-1 no c)
    R ra[M], rb[M], rc[M], rd[M];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int r = tid * M + j;
      ra[j] = r == 0 ? R(0) : buf[r];
      rb[j] = buf[NP + r];
      rc[j] = r == n - 1 ? R(0) : buf[2 * NP + r];
      rd[j] = buf[3 * NP + r];
    }
    __syncthreads();  // the row buffers are free: start loading the next system
    if (tid == 0 && s + (int)gridDim.x < nsys) issue(s + gridDim.x);
    // modified Thomas on the own rows: x_j + a'_j x_0 + c'_j x_{j+1} = d'_j ...
    R inv = fast_rcp(rb[1]);
    R ap = ra[1] * inv, cp = rc[1] * inv, dp = rd[1] * inv;
    ra[1] = ap; rc[1] = cp; rd[1] = dp;
#pragma unroll
    for (int j = 2; j < M; ++j) {
      const R aj = ra[j];
      const R r = fast_rcp(fmaT(-aj, cp, rb[j]));
      ap = -aj * ap * r;
      dp = fmaT(-aj, dp, rd[j]) * r;
      cp = rc[j] * r;
      ra[j] = ap; rc[j] = cp; rd[j] = dp;
    }
    // ... then x_j + a''_j x_0 + c''_j x_{M-1} = d''_j for j = 1..M-2
    R an = ra[M - 2], cn = rc[M - 2], dn = rd[M - 2];
#pragma unroll
    for (int j = M - 3; j >= 1; --j) {
      const R cj = rc[j];
      dn = fmaT(-cj, dn, rd[j]);
      an = fmaT(-cj, an, ra[j]);
      cn = -cj * cn;
      ra[j] = an; rc[j] = cn; rd[j] = dn;
    }
    const R r0 = fast_rcp(fmaT(-rc[0], an, rb[0]));
    const R eA = ra[0] * r0, eC = -rc[0] * cn * r0, eD = fmaT(-rc[0], dn, rd[0]) * r0;
    R x0, xl;
    reduced_pcr<R, kStreamT>(red, tid, true, eA, eC, eD, ap, cp, dp, x0, xl);
    // the previous solution must have left xbuf before it is overwritten
    if (tid == 0) bulk_store_wait_read();
    __syncthreads();
    xbuf[tid * M] = x0;
#pragma unroll
    for (int j = 1; j < M - 1; ++j) xbuf[tid * M + j] = fmaT(-rc[j], xl, fmaT(-ra[j], x0, rd[j]));
    xbuf[tid * M + M - 1] = xl;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> copy engine
    __syncthreads();
    if (tid == 0) bulk_store(x + (size_t)s * n, xbuf, bytes);
  }
  if (failed) {
    if (tid == 0) {
      atomicExch(&g_tri_timeout, 1);
      mbar_wait_bounded(bar, parity);  // copies still in flight land before the CTA leaves
    }
  }
  if (tid == 0) bulk_store_wait_all();
}

template <class R, int M>
cudaError_t stream_launch(const R* a, const R* b, const R* c, const R* d, R* x, int n, int nsys, cudaStream_t st) {
  auto k = tri_stream_kernel<R, M>;
  const size_t smem = stream_smem_bytes<R, M>();
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, nsm = 0, per_sm = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kStreamT, smem)) != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidValue;
  const int grid = std::min(nsys, nsm * per_sm);
  k<<<grid, kStreamT, smem, st>>>(a, b, c, d, x, n, nsys);
  return cudaGetLastError();
}

// The streamed kernel applies when the copies are legal (16-byte aligned
// system starts and sizes) and the rows fit one CTA: n <= 256*M for an odd
// M <= 19 whose buffers fit the shared memory.
template <class R>
bool stream_fits(const R* a, const R* b, const R* c, const R* d, const R* x, int n) {
  const uintptr_t all = (uintptr_t)a | (uintptr_t)b | (uintptr_t)c | (uintptr_t)d | (uintptr_t)x;
  if ((all & 15) != 0 || ((size_t)n * sizeof(R)) % 16 != 0) return false;
  return n >= 3 * kStreamT / 2 && n <= kStreamT * 19;
}

template <class R>
cudaError_t stream_solve(const R* a, const R* b, const R* c, const R* d, R* x, int n, int nsys, cudaStream_t st) {
  int m = (n + kStreamT - 1) / kStreamT;
  m |= 1;
  if (m < 3) m = 3;
  switch (m) {
    case 3: return stream_launch<R, 3>(a, b, c, d, x, n, nsys, st);
    case 5: return stream_launch<R, 5>(a, b, c, d, x, n, nsys, st);
    case 7: return stream_launch<R, 7>(a, b, c, d, x, n, nsys, st);
    case 9: return stream_launch<R, 9>(a, b, c, d, x, n, nsys, st);
    case 11: return stream_launch<R, 11>(a, b, c, d, x, n, nsys, st);
    case 13: return stream_launch<R, 13>(a, b, c, d, x, n, nsys, st);
    case 15: return stream_launch<R, 15>(a, b, c, d, x, n, nsys, st);
    case 17: return stream_launch<R, 17>(a, b, c, d, x, n, nsys, st);
    case 19: return stream_launch<R, 19>(a, b, c, d, x, n, nsys, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Interleaved systems (row i of system s at i*nsys + s), hybrid solver.
// A group of W adjacent systems occupies SEG = W*sizeof(R) contiguous bytes
// of every row: 128-byte segments stream from HBM at full rate, 64-byte ones
// a little below it and 32-byte ones (4 binary64 systems) at under 40 % of
// it.  A thread-block cluster of Q CTAs (one per SM) solves one group at a
// time, CTA q holding rows q*ROWS .. q*ROWS+ROWS-1 of all W systems: thread
// t owns rows k*16 .. k*16+15 (k = t / W) of system w = t % W.  Each group
// arrives as four tiles (a, b, c, d; boxes of W x 256 rows, copied by the
// tensor engine without multicast) in shared memory while the CTA is still
// solving the previous group from registers.  Every thread eliminates its
// 16 rows (modified Thomas) to two rows coupled to the neighbouring chunks.
// The reduced rows of system w are solved in cluster rank w % Q (its owner)
// by one warp (Thomas-PCR on 32 lanes): every CTA stages its reduced rows in
// the owners' layout and sends each owner its runs by bulk shared-to-shared
// copies that complete on the owner's mbarrier.  After a cluster barrier
// every thread reads its two solutions back and back-substitutes into a
// solution tile that the tensor engine stores.  The reduced rows are
// double-buffered across groups.  Every wait on a copy is bounded
// (g_tri_timeout, as above).  (SEG, ROWS) = (128, 256) for lines of up to
// 2048 rows; (64, 512) above, which halves W and so the cluster size that
// holds a 4096-row group (8 instead of 16 CTAs: more clusters fit the GPU).
// ---------------------------------------------------------------------------
namespace {

namespace cg = cooperative_groups;

constexpr int kStrM = 16;    // rows per thread
constexpr int kStrBox = 256;  // rows per 2-D tile box (the tensor-copy limit)

// A configuration: SEG bytes of every row per group (W = SEG / sizeof(R)
// systems) and ROWS rows per CTA, so that a cluster of Q CTAs covers
// Q * ROWS rows.  (128, 256): W = 16 / 32, clusters of up to 16 CTAs;
// (64, 512): W = 8 / 16, clusters of up to 8 (n <= 4096 in both).
template <class R, int SEG, int ROWS>
struct StridedCfg {
  static constexpr int W = SEG / (int)sizeof(R);  // systems per group
  static constexpr int C = ROWS / kStrM;          // chunks per CTA per system
  static constexpr int T = W * C;                 // threads per CTA
  static constexpr int TILE = W * ROWS;           // elements per tile
  static constexpr int BOXES = ROWS / kStrBox;    // tile boxes per array
  // The 2*C*Q reduced rows of a system are 32 lane chunks of m = C*Q/16
  // rows, at pitch m + 2 (even, so that a chunk's two reduced rows are one
  // aligned pair).  The owner of a system solves m rows per lane, so m is
  // 4, 8 or 16 (warp_unit_solve): Q <= QMAX.
  static constexpr int QMAX = (256 / C < W ? 256 / C : W) < 16 ? (256 / C < W ? 256 / C : W) : 16;
  // one set of gathered reduced rows: a | c | d of the W / Q owned systems,
  // W * (2C + 64 / Q) elements per array, at most W * (2C + 16) (Q = 4)
  static constexpr int SETA = W * (2 * C + 16);
  // a CTA's rows for one owned system of one owner are one run of (32 / Q)
  // lane chunks: 2C + 64 / Q elements, at most 2C + 16 (Q = 4); W runs per array
  static constexpr int RUN = 2 * C + 16;
};

// shared memory (bytes): 4 input tiles, the solution tile, 2 sets of
// gathered reduced rows, the outgoing runs, 3 mbarriers (tiles, 2 sets)
template <class R, int SEG, int ROWS>
__host__ __device__ constexpr size_t strided_smem_bytes() {
  using SC = StridedCfg<R, SEG, ROWS>;
  return ((size_t)5 * SC::TILE + 2 * 3 * (size_t)SC::SETA + 3 * (size_t)SC::W * SC::RUN) * sizeof(R) + 32;
}

__device__ __forceinline__ void tile_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tile_store_2d(const CUtensorMap* map, int x, int y, const void* src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(smem_u32(src))
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// shared::cluster address of `local`'s counterpart in cluster rank `rank`
__device__ __forceinline__ unsigned cluster_smem_addr(const void* local, int rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(local)), "r"(rank));
  return r;
}

// bulk copy from this CTA's shared memory to cluster shared memory,
// completing on the destination's mbarrier
__device__ __forceinline__ void bulk_send(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   dst),
               "r"(smem_u32(src)), "r"(bytes), "r"(bar)
               : "memory");
}

// One warp solves a system of 32*m rows (m >= 2) with unit diagonals:
// x_i + a_i x_{i-1} + c_i x_{i+1} = d_i, lane l's rows at l*pitch ..
// l*pitch+m-1 of the arrays a, c, d.  Each lane eliminates its rows to the
// first and last (modified Thomas, as in thomas_pcr_warp, its intermediate
// rows in the scratch arrays sa, sc, sd so that the inputs are only read),
// the 64 rows are solved by PCR over register shuffles, and each lane
// back-substitutes.  The solution replaces d.
template <class R, int m>
__device__ __forceinline__ void warp_unit_solve(const R* __restrict__ a, const R* __restrict__ c, R* __restrict__ d,
                                                R* __restrict__ sa, R* __restrict__ sc, R* __restrict__ sd,
                                                int pitch) {
  const int lane = threadIdx.x & 31;
  const R* la = a + lane * pitch;
  const R* lc = c + lane * pitch;
  R* ld = d + lane * pitch;
  R* xa = sa + lane * pitch;
  R* xc = sc + lane * pitch;
  R* xd = sd + lane * pitch;
  R eA, eC, eD, oA, oC, oD;
  if constexpr (m == 2) {
    eA = la[0]; eC = lc[0]; eD = ld[0];
    oA = la[1]; oC = lc[1]; oD = ld[1];
  } else {
    // forward: rows 1..m-1 -> x_k + a'_k x_0 + c'_k x_{k+1} = d'_k
    R ap = la[1], cp = lc[1], dp = ld[1];
    xa[1] = ap; xc[1] = cp; xd[1] = dp;
#pragma unroll
    for (int k = 2; k < m; ++k) {
      const R ak = la[k];
      const R r = fast_rcp(fmaT(-ak, cp, R(1)));
      ap = -ak * ap * r;
      dp = fmaT(-ak, dp, ld[k]) * r;
      cp = lc[k] * r;
      xa[k] = ap; xc[k] = cp; xd[k] = dp;
    }
    oA = ap; oC = cp; oD = dp;
    // backward: rows m-3..1 -> x_k + a''_k x_0 + c''_k x_{m-1} = d''_k
    R an = xa[m - 2], cn = xc[m - 2], dn = xd[m - 2];
#pragma unroll
    for (int k = m - 3; k >= 1; --k) {
      const R ck = xc[k];
      dn = fmaT(-ck, dn, xd[k]);
      an = fmaT(-ck, an, xa[k]);
      cn = -ck * cn;
      xa[k] = an; xc[k] = cn; xd[k] = dn;
    }
    const R c0 = lc[0];
    const R r0 = fast_rcp(fmaT(-c0, an, R(1)));
    eA = la[0] * r0; eC = -c0 * cn * r0; eD = fmaT(-c0, dn, ld[0]) * r0;
  }
  // PCR on the 64 interleaved rows (even: first rows, odd: last rows), unit
  // diagonals kept by normalising every step
  auto step = [](R& A, R& C, R& D, R lA, R lC, R lD, R hA, R hC, R hD) {
    const R r = fast_rcp(fmaT(-C, hA, fmaT(-A, lC, R(1))));
    const R nA = -A * lA * r, nC = -C * hC * r, nD = fmaT(-C, hD, fmaT(-A, lD, D)) * r;
    A = nA; C = nC; D = nD;
  };
  {  // row stride 1: even rows see the odd row of lane-1 and their own; odd rows their own even and lane+1's
    R lA = shfl_up_r(oA, 1), lC = shfl_up_r(oC, 1), lD = shfl_up_r(oD, 1);
    R hA = shfl_dn_r(eA, 1), hC = shfl_dn_r(eC, 1), hD = shfl_dn_r(eD, 1);
    if (lane == 0) { lA = R(0); lC = R(0); lD = R(0); }
    if (lane == 31) { hA = R(0); hC = R(0); hD = R(0); }
    const R e0A = eA, e0C = eC, e0D = eD;
    step(eA, eC, eD, lA, lC, lD, oA, oC, oD);
    step(oA, oC, oD, e0A, e0C, e0D, hA, hC, hD);
  }
#pragma unroll
  for (int dl = 1; dl < 32; dl <<= 1) {  // row stride 2*dl: same-parity rows of lanes +-dl
    R lEA = shfl_up_r(eA, dl), lEC = shfl_up_r(eC, dl), lED = shfl_up_r(eD, dl);
    R hEA = shfl_dn_r(eA, dl), hEC = shfl_dn_r(eC, dl), hED = shfl_dn_r(eD, dl);
    R lOA = shfl_up_r(oA, dl), lOC = shfl_up_r(oC, dl), lOD = shfl_up_r(oD, dl);
    R hOA = shfl_dn_r(oA, dl), hOC = shfl_dn_r(oC, dl), hOD = shfl_dn_r(oD, dl);
    if (lane < dl) { lEA = R(0); lEC = R(0); lED = R(0); lOA = R(0); lOC = R(0); lOD = R(0); }
    if (lane + dl > 31) { hEA = R(0); hEC = R(0); hED = R(0); hOA = R(0); hOC = R(0); hOD = R(0); }
    step(eA, eC, eD, lEA, lEC, lED, hEA, hEC, hED);
    step(oA, oC, oD, lOA, lOC, lOD, hOA, hOC, hOD);
  }
  const R x0 = eD, xl = oD;
  ld[0] = x0;
#pragma unroll
  for (int k = 1; k < m - 1; ++k) ld[k] = fmaT(-xc[k], xl, fmaT(-xa[k], x0, xd[k]));
  ld[m - 1] = xl;
}

// pairs of adjacent elements (16 bytes in binary64, 8 in binary32)
template <class R>
struct Pair2;
template <>
struct Pair2<double> { using type = double2; };
template <>
struct Pair2<float> { using type = float2; };

template <class R, int SEG, int ROWS>
__global__ void __launch_bounds__(StridedCfg<R, SEG, ROWS>::T, 1)
    tri_strided_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                       const __grid_constant__ CUtensorMap mapC, const __grid_constant__ CUtensorMap mapD,
                       const __grid_constant__ CUtensorMap mapX, int n, int nsys) {
  using SC = StridedCfg<R, SEG, ROWS>;
  using P2 = typename Pair2<R>::type;
  constexpr int W = SC::W, T = SC::T, M = kStrM, CH = SC::C;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* tile = reinterpret_cast<R*>(smem_raw);  // a | b | c | d, [row][system] each
  R* xt = tile + 4 * SC::TILE;               // solution tile
  R* sets = xt + SC::TILE;                   // 2 x (a | c | d), SETA each
  R* outr = sets + 2 * 3 * SC::SETA;         // outgoing runs: [array][w][RUN]
  uint64_t* bar = reinterpret_cast<uint64_t*>(outr + 3 * W * SC::RUN);  // tiles
  uint64_t* rbar = bar + 1;                                            // reduced rows of set 0, 1
  cg::cluster_group cluster = cg::this_cluster();
  const int Q = (int)cluster.num_blocks();  // 4 .. SC::QMAX, a power of two
  const int rank = (int)cluster.block_rank();
  const int S = W / Q;                       // systems each CTA owns
  const int m = CH * Q / 16;                 // reduced rows per lane chunk: 4, 8 or 16
  const int pitch = m + 2;                   // lane chunks of m reduced rows, padded
  const int sysP = 32 * pitch;               // one owned system in a set array
  const int run = (32 / Q) * pitch;          // this CTA's part of one owned system
  const int tid = threadIdx.x;
  const int w = tid % W, k = tid / W;
  const int owner = w % Q, slot = w / Q;  // system w's reduced rows: rank `owner`, slot `slot`
  const int row0 = rank * ROWS + k * M;
  const int nclusters = gridDim.x / Q;
  const int cl = blockIdx.x / Q;
  const int ngroups = (nsys + W - 1) / W;
  const bool stores = rank * ROWS < n;  // CTAs wholly past the last row store nothing
  // this chunk's reduced rows 2i, 2i+1 (i = rank*C + k): their pair in the
  // run for system w and in the owner's set (m and 2i are even: one lane
  // chunk, even position)
  const int i2 = 2 * (rank * CH + k);
  const int q_run = ((2 * k) / m) * pitch + (2 * k) % m;
  const int p_e = slot * sysP + (i2 / m) * pitch + i2 % m;
  // bytes an owner receives per group: Q senders x S systems x 3 arrays x run
  const unsigned recv_bytes = (unsigned)(3 * W * run * sizeof(R));
  constexpr unsigned kTileBytes = (unsigned)(SC::TILE * sizeof(R));
  auto issue = [&](int g) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier reads of the tiles precede the copies
    mbar_expect_tx(bar, 4 * kTileBytes);
#pragma unroll
    for (int bx = 0; bx < SC::BOXES; ++bx) {
      const int y = rank * ROWS + bx * kStrBox, o = bx * kStrBox * W;
      tile_load_2d(tile + o, &mapA, g * W, y, bar);
      tile_load_2d(tile + SC::TILE + o, &mapB, g * W, y, bar);
      tile_load_2d(tile + 2 * SC::TILE + o, &mapC, g * W, y, bar);
      tile_load_2d(tile + 3 * SC::TILE + o, &mapD, g * W, y, bar);
    }
  };
  if (tid == 0) {
    mbar_init(bar);
    mbar_init(rbar);
    mbar_init(rbar + 1);
  }
  cluster.sync();  // every CTA of the cluster runs and its mbarriers are set up
  if (tid == 0 && cl < ngroups) issue(cl);
  unsigned parity = 0, rpar = 0;
  bool failed = false;
  int set = 0;
  for (int g = cl; g < ngroups; g += nclusters, set ^= 1) {
    const int sys = g * W + w;
    const bool live = sys < nsys;
    if (tid == 0) mbar_expect_tx(rbar + set, recv_bytes);  // this group's reduced rows, from every CTA
    if (!failed) {
      const bool ok = mbar_wait_bounded(bar, parity);
      failed = __syncthreads_or(!ok);
      parity ^= 1;
    }
    // own rows into registers; row 0 has no a, row n-1 no c, and rows or
    // systems outside the problem (zeros in the tiles) become identity rows
    R ra[M], rb[M], rc[M], rd[M];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int o = (k * M + j) * W + w;
      ra[j] = tile[o];
      rb[j] = tile[SC::TILE + o];
      rc[j] = tile[2 * SC::TILE + o];
      rd[j] = tile[3 * SC::TILE + o];
    }
    if (!(live && row0 >= 1 && row0 + M <= n - 1)) {
#pragma unroll
      for (int j = 0; j < M; ++j) {
        const int r = row0 + j;
        if (!(live && r < n)) {
          ra[j] = R(0); rb[j] = R(1); rc[j] = R(0); rd[j] = R(0);
        } else {
          if (r == 0) ra[j] = R(0);
          if (r == n - 1) rc[j] = R(0);
        }
      }
    }
    __syncthreads();  // the tiles are free: start loading the cluster's next group
    if (tid == 0 && !failed && g + nclusters < ngroups) issue(g + nclusters);
    // modified Thomas on the own rows (as in the contiguous kernels)
    R inv = fast_rcp(rb[1]);
    R ap = ra[1] * inv, cp = rc[1] * inv, dp = rd[1] * inv;
    ra[1] = ap; rc[1] = cp; rd[1] = dp;
#pragma unroll
    for (int j = 2; j < M; ++j) {
      const R aj = ra[j];
      const R r = fast_rcp(fmaT(-aj, cp, rb[j]));
      ap = -aj * ap * r;
      dp = fmaT(-aj, dp, rd[j]) * r;
      cp = rc[j] * r;
      ra[j] = ap; rc[j] = cp; rd[j] = dp;
    }
    R an = ra[M - 2], cn = rc[M - 2], dn = rd[M - 2];
#pragma unroll
    for (int j = M - 3; j >= 1; --j) {
      const R cj = rc[j];
      dn = fmaT(-cj, dn, rd[j]);
      an = fmaT(-cj, an, ra[j]);
      cn = -cj * cn;
      ra[j] = an; rc[j] = cn; rd[j] = dn;
    }
    const R r0 = fast_rcp(fmaT(-rc[0], an, rb[0]));
    const R eA = ra[0] * r0, eC = -rc[0] * cn * r0, eD = fmaT(-rc[0], dn, rd[0]) * r0;
    // the chunk's reduced rows -> the run for its system, then every run to
    // its owner (the previous group's runs were read before its barrier)
    {
      P2* o = reinterpret_cast<P2*>(outr + w * SC::RUN + q_run);
      o[0] = P2{eA, ap};
      o[W * SC::RUN / 2] = P2{eC, cp};
      o[W * SC::RUN] = P2{eD, dp};
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> copy engine
    __syncthreads();
    R* own = sets + (size_t)set * 3 * SC::SETA;  // this group's set: a | c | d
    if (tid < 3 * W && !failed) {
      const int arr = tid / W, ws = tid % W;  // run of system ws, array arr
      const int dst = arr * SC::SETA + (ws / Q) * sysP + (32 / Q) * rank * pitch;
      bulk_send(cluster_smem_addr(own + dst, ws % Q), outr + (arr * W + ws) * SC::RUN,
                (unsigned)(run * sizeof(R)), cluster_smem_addr(rbar + set, ws % Q));
    }
    if (!failed) {
      const bool ok = mbar_wait_bounded(rbar + set, (rpar >> set) & 1u);
      failed = __syncthreads_or(!ok);
      rpar ^= 1u << set;
    }
    // one warp per owned system (S of them, 32Q rows each); the other set,
    // idle until this group's barrier, holds the intermediate rows
    {
      R* scr = sets + (size_t)(set ^ 1) * 3 * SC::SETA;
      for (int s = tid >> 5; s < S; s += T / 32) {
        const int o = s * sysP;
        R* A = own + o;
        R* Cc = own + SC::SETA + o;
        R* D = own + 2 * SC::SETA + o;
        R* sa = scr + o;
        R* sc = scr + SC::SETA + o;
        R* sd = scr + 2 * SC::SETA + o;
        switch (m) {
          case 4: warp_unit_solve<R, 4>(A, Cc, D, sa, sc, sd, pitch); break;
          case 8: warp_unit_solve<R, 8>(A, Cc, D, sa, sc, sd, pitch); break;
          default: warp_unit_solve<R, 16>(A, Cc, D, sa, sc, sd, pitch); break;
        }
      }
    }
    if (tid == 0) bulk_store_wait_read();  // the previous solution tile has been read out
    cluster.sync();
    const P2 sol = *reinterpret_cast<const P2*>(cluster.map_shared_rank(own + 2 * SC::SETA, owner) + p_e);
    const R x0 = sol.x, xl = sol.y;
#pragma unroll
    for (int j = 0; j < M; ++j)
      xt[(k * M + j) * W + w] = j == 0 ? x0 : (j == M - 1 ? xl : fmaT(-rc[j], xl, fmaT(-ra[j], x0, rd[j])));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor engine
    __syncthreads();
    // rows past n and systems past nsys fall outside the map and are not written
    if (tid == 0 && !failed && stores) {
#pragma unroll
      for (int bx = 0; bx < SC::BOXES; ++bx)
        if (rank * ROWS + bx * kStrBox < n) tile_store_2d(&mapX, g * W, rank * ROWS + bx * kStrBox, xt + bx * kStrBox * W);
    }
  }
  if (tid == 0) {
    if (failed) {
      atomicExch(&g_tri_timeout, 1);
      mbar_wait_bounded(bar, parity);  // copies still in flight land before the CTA leaves
      mbar_wait_bounded(rbar, rpar & 1u);
      mbar_wait_bounded(rbar + 1, (rpar >> 1) & 1u);
    }
    bulk_store_wait_all();
  }
  cluster.sync();  // no CTA leaves while another may still read its shared memory
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no
// link-time dependence on the driver library)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// [n rows][nsys systems] in boxes of W systems x 256 rows; rows and systems
// past the ends read as zeros and are not written
template <class R>
bool strided_map(CUtensorMap* map, const R* p, int n, int nsys, int W) {
  const EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)nsys, (cuuint64_t)n};
  const cuuint64_t strides[1] = {(cuuint64_t)nsys * sizeof(R)};
  const cuuint32_t box[2] = {(cuuint32_t)W, (cuuint32_t)kStrBox};
  const cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt = sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  return fn(map, dt, 2, const_cast<R*>(p), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// cudaErrorInvalidValue: outside the configuration's range (n above
// QMAX * ROWS rows, or no room for a cluster of Q CTAs)
template <class R, int SEG, int ROWS>
cudaError_t strided_launch(const R* a, const R* b, const R* c, const R* d, R* x, int n, int nsys, cudaStream_t st) {
  using SC = StridedCfg<R, SEG, ROWS>;
  int Q = 4;  // CTAs per cluster: a power of two >= 4 (W / Q systems of 32 lane chunks on each owner)
  while (Q * ROWS < n) Q <<= 1;
  if (Q > SC::QMAX) return cudaErrorInvalidValue;
  CUtensorMap maps[5];
  if (!strided_map(&maps[0], a, n, nsys, SC::W) || !strided_map(&maps[1], b, n, nsys, SC::W) ||
      !strided_map(&maps[2], c, n, nsys, SC::W) || !strided_map(&maps[3], d, n, nsys, SC::W) ||
      !strided_map(&maps[4], static_cast<const R*>(x), n, nsys, SC::W))
    return cudaErrorInvalidValue;
  auto k = tri_strided_kernel<R, SEG, ROWS>;
  const size_t smem = strided_smem_bytes<R, SEG, ROWS>();
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (Q > 8 && (e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess)
    return e;
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = Q;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(SC::T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(Q);
  int max_clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&max_clusters, k, &cfg) != cudaSuccess || max_clusters < 1) {
    cudaGetLastError();
    return cudaErrorInvalidValue;
  }
  const int ngroups = (nsys + SC::W - 1) / SC::W;
  cfg.gridDim = dim3(Q * std::min(ngroups, max_clusters));
  e = cudaLaunchKernelEx(&cfg, k, maps[0], maps[1], maps[2], maps[3], maps[4], n, nsys);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

// IXB_STRIDED_SEG=64 or 128 forces one configuration; otherwise lines of
// more than 2048 rows use 64-byte segments with 512-row CTAs (clusters of
// 8 instead of 16, so more of them fit the GPU at once), shorter lines
// 128-byte segments with 256-row CTAs (less padding).
int strided_seg_choice() {
  static const int v = [] {
    const char* e = std::getenv("IXB_STRIDED_SEG");
    return e ? std::atoi(e) : 0;
  }();
  return v;
}

// cudaErrorInvalidValue: outside the kernels' range (n > 4096 rows, a row
// pitch or base address the tensor copies cannot take, or no room for a
// cluster); the caller then uses the general interleaved kernel
template <class R>
cudaError_t strided_solve(const R* a, const R* b, const R* c, const R* d, R* x, int n, int nsys, cudaStream_t st) {
  if (n < 1 || n > 16 * kStrBox || nsys < 1) return cudaErrorInvalidValue;
  const uintptr_t all = (uintptr_t)a | (uintptr_t)b | (uintptr_t)c | (uintptr_t)d | (uintptr_t)x;
  if ((all & 15) != 0 || ((size_t)nsys * sizeof(R)) % 16 != 0) return cudaErrorInvalidValue;
  const int seg = strided_seg_choice();
  if (seg == 64 || (seg != 128 && n > 8 * kStrBox)) {
    const cudaError_t e = strided_launch<R, 64, 512>(a, b, c, d, x, n, nsys, st);
    if (e != cudaErrorInvalidValue) return e;
  }
  return strided_launch<R, 128, 256>(a, b, c, d, x, n, nsys, st);
}

}  // namespace

template <class R, int SOLVER, int TL>
static cudaError_t contig_tl(const R* a, const R* b, const R* c, const R* d, R* x, int n, int nsys, int m, int mp,
                             size_t smem, cudaStream_t st) {
  auto k = tri_contig_kernel<R, SOLVER, TL, 256 / TL>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int grid = (nsys + TL - 1) / TL;
  k<<<grid, 256, smem, st>>>(a, b, c, d, x, n, nsys, m, mp);
  return cudaGetLastError();
}

template <class R, int SOLVER>
static cudaError_t tridiag_impl(const R* a, const R* b, const R* c, const R* d, R* x, int n, int nsys, int layout,
                                cudaStream_t st) {
  if (layout == 0) {
    if (SOLVER == IXB_SOLVER_HYBRID && stream_fits(a, b, c, d, x, n)) {
      const cudaError_t e = stream_solve(a, b, c, d, x, n, nsys, st);
      if (e != cudaErrorInvalidValue) return e;  // otherwise: does not fit this GPU, use the staged kernel
    }
    int g = 32;
    while (g < 256 && 3 * g < n) g <<= 1;
    const int tl = 256 / g;
    const int m = std::max(3, (n + g - 1) / g);
    const int mp = m | 1;
    const size_t smem = line_smem_elems(g, mp) * sizeof(R) * tl;
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem > (size_t)optin) return cudaErrorInvalidValue;  // line too long for one CTA
    switch (tl) {
      case 1: return contig_tl<R, SOLVER, 1>(a, b, c, d, x, n, nsys, m, mp, smem, st);
      case 2: return contig_tl<R, SOLVER, 2>(a, b, c, d, x, n, nsys, m, mp, smem, st);
      case 4: return contig_tl<R, SOLVER, 4>(a, b, c, d, x, n, nsys, m, mp, smem, st);
      default: return contig_tl<R, SOLVER, 8>(a, b, c, d, x, n, nsys, m, mp, smem, st);
    }
  }
  if (SOLVER == IXB_SOLVER_HYBRID) {
    const cudaError_t es = strided_solve(a, b, c, d, x, n, nsys, st);
    if (es != cudaErrorInvalidValue) return es;  // otherwise: size outside the cluster kernel's range
  }
  R* work = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&work, (size_t)n * nsys * sizeof(R), st);
  if (e != cudaSuccess) return e;
  tri_inter_kernel<R, SOLVER><<<(nsys + 127) / 128, 128, 0, st>>>(a, b, c, d, x, work, n, nsys);
  e = cudaGetLastError();
  cudaError_t e2 = cudaFreeAsync(work, st);
  return e != cudaSuccess ? e : e2;
}

// Reads and clears the timeout flag the streamed and interleaved kernels set
// when a bounded wait on their copies expires (synchronous).
cudaError_t tridiag_take_timeout(int* flag) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_tri_timeout, sizeof(int));
  if (e != cudaSuccess) return e;
  if (v) {
    const int zero = 0;
    if ((e = cudaMemcpyToSymbol(g_tri_timeout, &zero, sizeof(int))) != cudaSuccess) return e;
  }
  *flag = v;
  return cudaSuccess;
}

cudaError_t tridiag_set_first_wait_polls(int polls) {
  const int v = polls < 0 ? kSpinLimit : polls;
  return cudaMemcpyToSymbol(g_tri_first_wait_polls, &v, sizeof(int));
}

cudaError_t tridiag_f64(const double* a, const double* b, const double* c, const double* d, double* x, int n,
                        int nsys, int layout, int solver, cudaStream_t st) {
  if (solver == IXB_SOLVER_EXACT) return tridiag_impl<double, IXB_SOLVER_EXACT>(a, b, c, d, x, n, nsys, layout, st);
  return tridiag_impl<double, IXB_SOLVER_HYBRID>(a, b, c, d, x, n, nsys, layout, st);
}

cudaError_t tridiag_f32(const float* a, const float* b, const float* c, const float* d, float* x, int n, int nsys,
                        int layout, int solver, cudaStream_t st) {
  if (solver == IXB_SOLVER_EXACT) return tridiag_impl<float, IXB_SOLVER_EXACT>(a, b, c, d, x, n, nsys, layout, st);
  return tridiag_impl<float, IXB_SOLVER_HYBRID>(a, b, c, d, x, n, nsys, layout, st);
}

}  // namespace ixb

// ===========================================================================
// Allocation-free variant of ixb_tridiag_f64.
//
// Some callers cannot let a library allocate device memory while they run:
// a Fortran driver whose GPU memory is owned by its OpenACC runtime or by a
// pool it reserved at start-up, a solver sharing a GPU under a fixed memory
// budget where an allocation in mid-run can fail, or a loop that must not
// pay the implicit synchronisation that cudaMalloc/cudaFree may cause.  For
// them, the interleaved layout keeps its scratch in a fixed array that is
// part of this library's device image (allocated by the driver together
// with the library's code, once per GPU, and held until the process exits).
// ===========================================================================
namespace ixb {
namespace {

// Scratch of the interleaved solve: IXB_NOALLOC_MAX_ELEMS doubles (8 MiB).
__device__ __align__(256) double g_noalloc_scratch[IXB_NOALLOC_MAX_ELEMS];

constexpr int kMaxDevices = 64;
double* g_noalloc_ptr[kMaxDevices] = {};
std::mutex g_noalloc_mutex;

// Device address of the scratch array for the current device.  In host code
// the name g_noalloc_scratch denotes a host-side shadow, not device memory,
// so the address is looked up with that device current.  Outside stream
// capture it is looked up on every call (a context destroyed and re-created,
// e.g. after cudaDeviceReset, reloads the module at another address); while
// `st` is capturing, the address of the last uncaptured call on this device
// is used, so the first call on a device must come before any capture.
cudaError_t noalloc_scratch(cudaStream_t st, double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  } else if (!g_noalloc_ptr[dev]) {
    return cudaErrorStreamCaptureUnsupported;
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

}  // namespace
}  // namespace ixb

extern "C" int ixb_tridiag_f64_noalloc(const double* a, const double* b, const double* c, const double* d, double* x,
                                       int n, int nsys, int layout, int solver, void* stream) {
  using namespace ixb;
  if (!a || !b || !c || !d || !x || n < 1 || nsys < 1 || (layout != 0 && layout != 1)) return IXB_EINVAL;
  if (solver != IXB_SOLVER_HYBRID && solver != IXB_SOLVER_EXACT) return IXB_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (layout == 0) {
    // contiguous systems are staged in shared memory: no scratch at all
    e = solver == IXB_SOLVER_EXACT ? tridiag_impl<double, IXB_SOLVER_EXACT>(a, b, c, d, x, n, nsys, 0, st)
                                   : tridiag_impl<double, IXB_SOLVER_HYBRID>(a, b, c, d, x, n, nsys, 0, st);
  } else {
    if ((size_t)n * (size_t)nsys > (size_t)IXB_NOALLOC_MAX_ELEMS) return IXB_EINVAL;
    double* work = nullptr;
    e = noalloc_scratch(st, &work);
    if (e == cudaSuccess) {
      // every work[] element is written before it is read: nothing to clear
      if (solver == IXB_SOLVER_EXACT)
        tri_inter_kernel<double, IXB_SOLVER_EXACT><<<(nsys + 127) / 128, 128, 0, st>>>(a, b, c, d, x, work, n, nsys);
      else
        tri_inter_kernel<double, IXB_SOLVER_HYBRID><<<(nsys + 127) / 128, 128, 0, st>>>(a, b, c, d, x, work, n, nsys);
      e = cudaGetLastError();
    }
  }
  if (e == cudaErrorInvalidValue) return IXB_EINVAL;
  return e == cudaSuccess ? IXB_OK : IXB_ECUDA;
}

// Failure-detection hook (no counterpart in the reference): the poll limit of
// the first copy wait of every CTA of the streamed contiguous solve.
extern "C" int ixb_tridiag_set_first_wait_limit(int polls) {
  return ixb::tridiag_set_first_wait_polls(polls) == cudaSuccess ? IXB_OK : IXB_ECUDA;
}
