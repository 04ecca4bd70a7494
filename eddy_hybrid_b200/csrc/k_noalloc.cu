// k_noalloc.cu -- max |div u| over the interior with no device allocation.
//
// Some callers cannot call cudaMalloc: a Fortran time loop whose memory is
// owned by another framework's allocator, code running inside a region where
// allocation is forbidden, or a host program that only holds raw device
// pointers and no solver context.  eddy_max_divergence needs a context (its
// partial results live in context-owned scratch); this variant keeps its
// scratch in a fixed file-scope device array instead, so the caller passes
// only the fields, the metric arrays and an output slot.
//
// The scratch array is loaded with the library on every GPU that loads it and
// stays there until the process exits.  Its size caps the grid this entry
// point accepts (EDDY_NOALLOC_MAX_CELLS in include/eddy_b200.h).
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/eddy_b200.h"

namespace {

constexpr int kCellsPerBlock = 4096;                                     // interior cells reduced per block
constexpr int kMaxPartials = EDDY_NOALLOC_MAX_CELLS / kCellsPerBlock;    // 65536 partials (512 KiB)
static_assert(EDDY_NOALLOC_MAX_CELLS % kCellsPerBlock == 0, "scratch sizing");

// Per-block partial maxima.  Shared by every call: each call writes exactly
// the slots it later reads, so nothing has to be cleared between calls, but
// two calls that overlap on the GPU (different streams, no ordering) race on
// these slots.
static __device__ __align__(256) double g_divmax_partials[kMaxPartials];

// Device address of the scratch array per CUDA context.  A __device__
// array's address belongs to the context the module was loaded into, so the
// cache is keyed by the current context (the primary context of a device in
// the runtime API; a driver-API caller may have made another one current).
constexpr int kMaxContexts = 64;
std::mutex g_mu;
struct ScratchEntry {
  void *cuctx;
  double *addr;
};
ScratchEntry g_scratch[kMaxContexts] = {};
int g_nscratch = 0;

typedef int (*CtxGetCurrentFn)(void **);

__global__ void __launch_bounds__(256)
    k_divmax_partial(int nx, int ny, int nz, const double *__restrict__ u, const double *__restrict__ v,
                     const double *__restrict__ w, const double *__restrict__ ap, const double *__restrict__ bp,
                     const double *__restrict__ cp, long long ninner, double *__restrict__ part) {
  __shared__ double sh[256];
  const long long mi = nx - 2, mj = ny - 2;
  const long long sy = nx, sz = (long long)nx * ny;
  long long t0 = (long long)blockIdx.x * kCellsPerBlock;
  double mx = 0.;
  for (int r = threadIdx.x; r < kCellsPerBlock; r += blockDim.x) {
    long long t = t0 + r;
    if (t >= ninner) break;
    int i = 2 + (int)(t % mi), j = 2 + (int)((t / mi) % mj), k = 2 + (int)(t / (mi * mj));
    long long q = (i - 1) + sy * (j - 1) + sz * (k - 1);
    // DIVERGENCE, src/timeindeg.f:941-949 (ap, bp, cp are 1-based: entry i-1)
    double dv = (ap[i - 1] * (u[q] - u[q - 1]) + bp[j - 1] * (v[q] - v[q - sy]) + cp[k - 1] * (w[q] - w[q - sz]));
    mx = fmax(mx, fabs(dv));
  }
  sh[threadIdx.x] = mx;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(256) k_divmax_final(int nparts, const double *__restrict__ part, double *out) {
  __shared__ double sh[256];
  double mx = 0.;
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) mx = fmax(mx, part[b]);
  sh[threadIdx.x] = mx;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sh[0];
}

// Look up (once per context) the device address of the scratch array for
// the context current on this thread; host code cannot use the array's name
// as a device address.
int scratch_for_current_context(double **out) {
  static CtxGetCurrentFn get_ctx = nullptr;
  static bool resolved = false;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!resolved) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_ctx = reinterpret_cast<CtxGetCurrentFn>(p);
    resolved = true;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return EDDY_ECUDA;
  // make the device's primary context current if the thread has none yet
  if (cudaFree(nullptr) != cudaSuccess) return EDDY_ECUDA;
  void *cuctx = nullptr;
  if (!get_ctx || get_ctx(&cuctx) != 0 || !cuctx) return EDDY_ECUDA;
  for (int e = 0; e < g_nscratch; e++)
    if (g_scratch[e].cuctx == cuctx) {
      *out = g_scratch[e].addr;
      return EDDY_OK;
    }
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_divmax_partials) != cudaSuccess || !p) return EDDY_ECUDA;
  if (g_nscratch < kMaxContexts) g_scratch[g_nscratch++] = ScratchEntry{cuctx, static_cast<double *>(p)};
  *out = static_cast<double *>(p);
  return EDDY_OK;
}

}  // namespace

extern "C" int eddy_max_divergence_noalloc(int nx, int ny, int nz, const double *u, const double *v,
                                           const double *w, const double *ap, const double *bp, const double *cp,
                                           double *out, void *stream) {
  if (nx < 3 || ny < 3 || nz < 3 || !u || !v || !w || !ap || !bp || !cp || !out) return EDDY_EINVAL;
  long long ninner = (long long)(nx - 2) * (ny - 2) * (nz - 2);
  long long ncell = (long long)nx * ny * nz;
  if (ncell > (long long)EDDY_NOALLOC_MAX_CELLS) return EDDY_EINVAL;  // beyond the fixed scratch
  double *part = nullptr;
  int rc = scratch_for_current_context(&part);
  if (rc != EDDY_OK) return rc;
  // a launch error still pending on this thread from earlier work is cleared
  // here, so the checks below report this entry point's own launches only
  (void)cudaGetLastError();
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int nparts = (int)((ninner + kCellsPerBlock - 1) / kCellsPerBlock);
  k_divmax_partial<<<nparts, 256, 0, st>>>(nx, ny, nz, u, v, w, ap, bp, cp, ninner, part);
  if (cudaGetLastError() != cudaSuccess) return EDDY_ECUDA;
  k_divmax_final<<<1, 256, 0, st>>>(nparts, part, out);
  if (cudaGetLastError() != cudaSuccess) return EDDY_ECUDA;
  return EDDY_OK;
}
