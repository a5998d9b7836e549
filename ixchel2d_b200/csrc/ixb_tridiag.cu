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
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "ixb_internal.h"

namespace ixb {

template <class R, int SOLVER, int TL, int G>
__global__ void __launch_bounds__(TL * G) tri_contig_kernel(const R* __restrict__ a, const R* __restrict__ b,
                                                            const R* __restrict__ c, const R* __restrict__ d,
                                                            R* x, int n, int nsys, int m, int mp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
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
