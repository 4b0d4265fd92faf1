// LDA exchange-correlation without any device allocation.
//
// psc_lda_xc needs a context, and creating one allocates device memory.
// Some callers cannot allocate: code that is being captured into a CUDA graph
// (cudaMalloc is not a capturable operation), or hosts that hand every byte of
// device memory to their own pool allocator up front.  psc_lda_xc_noalloc
// serves them: it needs no context, and its only scratch -- one partial sum,
// maximum and minimum per CTA -- lives in the file-scope device array
// g_xc_scratch below (3 * PSC_XC_NOALLOC_MAX_CTAS doubles = 96 KiB), which
// every GPU that loads this library holds until the process exits.
//
// Set-up: the first call on a device looks up the device address of
// g_xc_scratch with cudaGetSymbolAddress (with that device current) and
// caches it; make that first call before any stream capture (a first call
// made during a capture is refused with status 2).  The cached address
// belongs to the device's primary context: a process that resets the device
// (cudaDeviceReset) must not call this entry point afterwards.  The minimum
// and maximum density propagate NaN, as numpy's max and min do.  Every call
// shares the one array, so calls that overlap on the GPU (two streams, or two
// host threads) race on it and must be serialised by the caller.  Each call
// writes every partial it later reads, so nothing has to be cleared between
// calls.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <mutex>

#define PSC_XC_NOALLOC_CHUNK 8192      // grid points per CTA
#define PSC_XC_NOALLOC_MAX_CTAS 4096   // => at most 33,554,432 points per call

static __device__ __align__(256) double g_xc_scratch[3 * PSC_XC_NOALLOC_MAX_CTAS];

namespace {

std::mutex g_mu;
double* g_scratch_dev[64] = {nullptr};  // device address of g_xc_scratch, per device

}  // namespace

// one CTA per chunk of PSC_XC_NOALLOC_CHUNK points
__global__ void __launch_bounds__(256)
k_xc_noalloc(const double* __restrict__ rho, double* __restrict__ vxc, long n, double* __restrict__ scratch) {
  __shared__ double sh[8];
  __shared__ double smx[8], smn[8];
  const long lo = (long)blockIdx.x * PSC_XC_NOALLOC_CHUNK;
  const long hi = min(n, lo + PSC_XC_NOALLOC_CHUNK);
  double e = 0.0, mx = -1e300, mn = 1e300;
  for (long i = lo + threadIdx.x; i < hi; i += 256) {
    const double r = rho[i];
    mx = psc_nanmax(mx, r);
    mn = psc_nanmin(mn, r);
    vxc[i] = psc_lda_point(r, e);
  }
  e = psc_block_sum<double, 256>(e, sh);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = psc_nanmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mn = psc_nanmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  }
  if ((threadIdx.x & 31) == 0) { smx[threadIdx.x >> 5] = mx; smn[threadIdx.x >> 5] = mn; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; ++w) { mx = psc_nanmax(mx, smx[w]); mn = psc_nanmin(mn, smn[w]); }
    scratch[blockIdx.x] = e;
    scratch[PSC_XC_NOALLOC_MAX_CTAS + blockIdx.x] = mx;
    scratch[2 * PSC_XC_NOALLOC_MAX_CTAS + blockIdx.x] = mn;
  }
}

__global__ void k_xc_noalloc_final(const double* __restrict__ scratch, int nblk, double h3, double* __restrict__ out) {
  __shared__ double sh[8];
  double s = 0.0;
  for (int i = threadIdx.x; i < nblk; i += 256) s += scratch[i];
  s = psc_block_sum<double, 256>(s, sh);
  if (threadIdx.x == 0) {
    double mx = -1e300, mn = 1e300;
    for (int i = 0; i < nblk; ++i) {
      mx = psc_nanmax(mx, scratch[PSC_XC_NOALLOC_MAX_CTAS + i]);
      mn = psc_nanmin(mn, scratch[2 * PSC_XC_NOALLOC_MAX_CTAS + i]);
    }
    out[0] = s * h3;
    out[1] = mx;
    out[2] = mn;
  }
}

extern "C" int psc_lda_xc_noalloc(const double* rho, double* vxc, long n, double h3, double* out_dev,
                                  void* stream) {
  if (!rho || !vxc || !out_dev) {
    psc_set_error(nullptr, "psc_lda_xc_noalloc: NULL pointer argument");
    return 2;
  }
  if (n < 1 || n > (long)PSC_XC_NOALLOC_CHUNK * PSC_XC_NOALLOC_MAX_CTAS) {
    psc_set_error(nullptr, "psc_lda_xc_noalloc: n must be between 1 and 33554432 grid points (the size of its "
                           "static scratch); use psc_lda_xc for larger grids");
    return 2;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    psc_set_error(nullptr, std::string("psc_lda_xc_noalloc: no usable current device: ") + cudaGetErrorString(e));
    return 1;
  }
  cudaStream_t st = (cudaStream_t)stream;
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_dev[dev]) {
      // the address lookup may load the module: it must not happen inside a
      // stream capture
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      e = cudaStreamIsCapturing(st, &cs);
      if (e != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        psc_set_error(nullptr, "psc_lda_xc_noalloc: the first call on a device sets up the scratch address and "
                               "must come before any stream capture");
        return 2;
      }
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_xc_scratch);
      if (e != cudaSuccess || !p) {
        psc_set_error(nullptr, std::string("psc_lda_xc_noalloc: cudaGetSymbolAddress failed: ") +
                                   cudaGetErrorString(e));
        return 1;
      }
      g_scratch_dev[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_dev[dev];
  }
  const int nblk = (int)((n + PSC_XC_NOALLOC_CHUNK - 1) / PSC_XC_NOALLOC_CHUNK);
  k_xc_noalloc<<<nblk, 256, 0, st>>>(rho, vxc, n, scratch);
  PSC_LAUNCH_CHECK((psc_ctx*)nullptr);
  k_xc_noalloc_final<<<1, 256, 0, st>>>(scratch, nblk, h3, out_dev);
  PSC_LAUNCH_CHECK((psc_ctx*)nullptr);
  return 0;
}
