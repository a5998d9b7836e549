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
// y-lines of a column-major field): one thread per system walks the rows;
// consecutive threads touch consecutive addresses.  The forward sweep keeps
// its modified diagonal (exact) or normalised super-diagonal (hybrid) in a
// scratch array of n*nsys elements taken from the stream-ordered allocator,
// and the modified right-hand side in x.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
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

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  for (int i = 0; i < kSpinLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
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
  unsigned parity = 0;
  bool failed = false;
  for (int s = blockIdx.x; s < nsys; s += gridDim.x) {
    const bool ok = mbar_wait_bounded(bar, parity);
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
// Interleaved systems (row i of system s at i*nsys + s), hybrid solver: a
// thread-block cluster of Q CTAs solves W adjacent systems at a time, CTA q
// holding rows q*R .. q*R+R-1 (R = (T/W)*M) of all W systems.  Thread t owns
// rows k*M .. k*M+M-1 (k = t / W) of system w = t % W, so a warp's loads and
// stores cover 32/W rows of W adjacent systems: whole 32-byte sectors.  Each
// thread eliminates its rows in registers (modified Thomas) to two rows; the
// 2*Q*(T/W) reduced rows of system w are gathered in the shared memory of
// cluster rank w (distributed shared memory) and solved there by PCR; every
// thread reads its two solutions back and back-substitutes.  The reduced
// rows are double-buffered across system groups, so a group costs two
// cluster barriers.  No bulk copies: plain coalesced loads from registers of
// several resident clusters per SM keep the memory system busy.
// ---------------------------------------------------------------------------
namespace {

namespace cg = cooperative_groups;

template <int W, int T, int M>
struct StridedShape {
  static constexpr int C = T / W;  // chunks per CTA per system
  static constexpr int R = C * M;  // rows per CTA
};

// reduced-row buffers of one CTA: 2 sets x ((a | c | d) x NR gathered rows
// + the PCR buffers of T threads)
template <class R>
__host__ __device__ constexpr size_t strided_set_elems(int nr, int t) {
  return (size_t)3 * nr + (size_t)12 * t;
}
template <class R>
__host__ __device__ constexpr size_t strided_smem_bytes(int nr, int t) {
  return 2 * strided_set_elems<R>(nr, t) * sizeof(R);
}

template <class R, int W, int T, int M>
__global__ void __launch_bounds__(T) tri_strided_kernel(const R* __restrict__ a, const R* __restrict__ b,
                                                        const R* __restrict__ c, const R* __restrict__ d,
                                                        R* __restrict__ x, int n, int nsys) {
  using SS = StridedShape<W, T, M>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* sm = reinterpret_cast<R*>(smem_raw);
  cg::cluster_group cluster = cg::this_cluster();
  const int Q = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int NR = 2 * Q * SS::C;  // reduced rows per system
  const int tid = threadIdx.x;
  const int w = tid % W, k = tid / W;
  const int row0 = rank * SS::R + k * M;
  const int nclusters = gridDim.x / Q;
  const int cl = blockIdx.x / Q;
  const int ngroups = (nsys + W - 1) / W;
  int set = 0;
  for (int g = cl; g < ngroups; g += nclusters, set ^= 1) {
    const int sys = g * W + w;
    const bool live = sys < nsys;
    R ra[M], rb[M], rc[M], rd[M];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int r = row0 + j;
      const bool in = live && r < n;
      const size_t o = (size_t)(in ? r : 0) * nsys + (live ? sys : 0);
      ra[j] = (in && r > 0) ? __ldg(a + o) : R(0);
      rb[j] = in ? __ldg(b + o) : R(1);
      rc[j] = (in && r < n - 1) ? __ldg(c + o) : R(0);
      rd[j] = in ? __ldg(d + o) : R(0);
    }
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
    // reduced rows 2i, 2i+1 (i = rank*C + k) of system w -> shared memory of rank w
    R* base = sm + (size_t)set * strided_set_elems<R>(NR, T);  // this set: a | c | d, then PCR buffers
    {
      R* dst = cluster.map_shared_rank(base, w % Q);
      const int i = 2 * (rank * SS::C + k);
      dst[i] = eA; dst[NR + i] = eC; dst[2 * NR + i] = eD;
      dst[i + 1] = ap; dst[NR + i + 1] = cp; dst[2 * NR + i + 1] = dp;
    }
    cluster.sync();
    if (rank < W) {  // owner of system `rank` of this group: solve its NR reduced rows
      // every thread takes RPT consecutive rows (padding rows beyond NR are
      // identity rows, decoupled); with 4 rows it first eliminates its two
      // middle rows (modified Thomas on 4 rows), so the PCR runs on 2 rows
      // per thread
      constexpr int RPT = 16 / W;  // NR / T: 4 (binary64, W = 4) or 2 (binary32, W = 8)
      R ea[RPT], ec[RPT], ed[RPT];
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        const int i = RPT * tid + q;
        const bool in = i < NR;
        ea[q] = in ? base[i] : R(0);
        ec[q] = in ? base[NR + i] : R(0);
        ed[q] = in ? base[2 * NR + i] : R(0);
      }
      R eA, eC, eD, oA, oC, oD, x0, xl;
      R m1a = R(0), m1c = R(0), m1d = R(0), m2a = R(0), m2c = R(0), m2d = R(0);
      if constexpr (RPT == 4) {
        // forward: rows 1..3 -> x_k + a'_k x_0 + c'_k x_{k+1} = d'_k (unit diagonals)
        R ap = ea[1], cp = ec[1], dp = ed[1];
        m1a = ap; m1c = cp; m1d = dp;
        R r = fast_rcp(fmaT(-ea[2], cp, R(1)));
        ap = -ea[2] * ap * r; dp = fmaT(-ea[2], dp, ed[2]) * r; cp = ec[2] * r;
        m2a = ap; m2c = cp; m2d = dp;
        r = fast_rcp(fmaT(-ea[3], cp, R(1)));
        oA = -ea[3] * ap * r; oD = fmaT(-ea[3], dp, ed[3]) * r; oC = ec[3] * r;
        // backward: row 1 -> x_1 + a''_1 x_0 + c''_1 x_3 = d''_1
        const R dn = fmaT(-m1c, m2d, m1d), an = fmaT(-m1c, m2a, m1a), cn = -m1c * m2c;
        m1a = an; m1c = cn; m1d = dn;
        const R r0 = fast_rcp(fmaT(-ec[0], an, R(1)));
        eA = ea[0] * r0; eC = -ec[0] * cn * r0; eD = fmaT(-ec[0], dn, ed[0]) * r0;
      } else {
        eA = ea[0]; eC = ec[0]; eD = ed[0];
        oA = ea[RPT - 1]; oC = ec[RPT - 1]; oD = ed[RPT - 1];
      }
      reduced_pcr<R, T>(base + 3 * NR, tid, true, eA, eC, eD, oA, oC, oD, x0, xl);
      // solutions of the owned rows -> base[2*NR + i], where the other CTAs read them
      if (RPT * tid < NR) {
        base[2 * NR + RPT * tid] = x0;
        if constexpr (RPT == 4) {
          base[2 * NR + 4 * tid + 1] = fmaT(-m1c, xl, fmaT(-m1a, x0, m1d));
          base[2 * NR + 4 * tid + 2] = fmaT(-m2c, xl, fmaT(-m2a, x0, m2d));
        }
        base[2 * NR + RPT * tid + RPT - 1] = xl;
      }
    }
    cluster.sync();
    // solutions of the own reduced rows, from rank w
    const R* sol = cluster.map_shared_rank(base + 2 * NR, w % Q);
    const int i = 2 * (rank * SS::C + k);
    const R x0 = sol[i], xl = sol[i + 1];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int r = row0 + j;
      if (live && r < n) {
        const R xv = j == 0 ? x0 : (j == M - 1 ? xl : fmaT(-rc[j], xl, fmaT(-ra[j], x0, rd[j])));
        x[(size_t)r * nsys + sys] = xv;
      }
    }
  }
  cluster.sync();  // no CTA leaves while another may still read its shared memory
}

template <class R, int W, int T, int M>
cudaError_t strided_launch(const R* a, const R* b, const R* c, const R* d, R* x, int n, int nsys, cudaStream_t st) {
  using SS = StridedShape<W, T, M>;
  const int Q = (n + SS::R - 1) / SS::R;
  if (Q < W || Q > 8) return cudaErrorInvalidValue;  // one owner CTA per system of a group
  const int nr = 2 * Q * SS::C;
  const size_t smem = strided_smem_bytes<R>(nr, T);
  auto k = tri_strided_kernel<R, W, T, M>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = Q;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(Q);
  int max_clusters = 0;
  if ((e = cudaOccupancyMaxActiveClusters(&max_clusters, k, &cfg)) != cudaSuccess) return e;
  if (max_clusters < 1) return cudaErrorInvalidValue;
  const int ngroups = (nsys + W - 1) / W;
  cfg.gridDim = dim3(Q * std::min(ngroups, max_clusters));
  e = cudaLaunchKernelEx(&cfg, k, a, b, c, d, x, n, nsys);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

// binary64: 4 systems (one 32-byte sector per row) x 32 chunks of 16 rows
// per CTA of 128 threads; binary32: 8 systems x 32 chunks of 16 rows per
// CTA of 256 threads.  Both cover up to 8 x 512 = 4096 rows per system.
template <class R>
cudaError_t strided_solve(const R* a, const R* b, const R* c, const R* d, R* x, int n, int nsys, cudaStream_t st) {
  if constexpr (sizeof(R) == 8) return strided_launch<R, 4, 128, 16>(a, b, c, d, x, n, nsys, st);
  else return strided_launch<R, 8, 256, 16>(a, b, c, d, x, n, nsys, st);
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
// so the address is looked up once per device with that device current.
cudaError_t noalloc_scratch(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = static_cast<double*>(p);
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
    e = noalloc_scratch(&work);
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
