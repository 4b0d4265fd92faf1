// Device building blocks of the Type-II multisecant mixer (Anderson mixing
// for group size 0), Mixer/msecant2.py:24-93.  The mixer's control flow -- the
// restart test, the EN stages, the groups, the quasi-inverse of the last
// group's r x r Gram matrix -- runs on the host; every operation on the
// n-vectors of the history (one column per SCF iteration, FP64, in HBM) is
// one of these:
//   psc_mix2_diff       df = f1 - df, dx = (x1 - dx) + mix df     (msecant2.py:58-60)
//   psc_mix2_store      dx = x1, df = f1                           (first call, restart, append)
//   psc_block_dots      c_i = A_i . x for the r columns of A       (DF^T df, DF^T f1)
//   psc_block_combine   y = base + mix f - sum_i A_i c_i           (the new iterate, DX updates)
//   psc_block_absrow_max max_p sum_i |A_i[p]|                       (the inf-norm of qinv.py:27)
// The Gram matrix of the last group and the block product DF C go through
// psc_gram and psc_gemm_nn.  Sums are deterministic (fixed partial counts and
// orders).
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>
#include <vector>

namespace {
constexpr int MX_NT = 256;
constexpr int MX_COEF = 256;   // coefficients per combine launch (staged in shared memory)
}  // namespace

__global__ void k_mix2_diff(const double* __restrict__ x1, const double* __restrict__ f1, double* __restrict__ dx,
                            double* __restrict__ df, double mix, long n) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    const double d = f1[p] - df[p];
    df[p] = d;
    dx[p] = (x1[p] - dx[p]) + mix * d;
  }
}

__global__ void k_mix2_store(const double* __restrict__ x1, const double* __restrict__ f1, double* __restrict__ dx,
                             double* __restrict__ df, long n) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    dx[p] = x1[p];
    df[p] = f1[p];
  }
}

// y = base + mix f - sum_{i < r} A_i c_i (f may be NULL; y may alias base)
__global__ void __launch_bounds__(MX_NT)
k_block_combine(double* y, const double* base, const double* __restrict__ f, double mix,
                const double* __restrict__ A, long lda, int r, const double* __restrict__ c, long n) {
  __shared__ double cs[MX_COEF];
  for (int i = threadIdx.x; i < r; i += MX_NT) cs[i] = c[i];
  __syncthreads();
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    double v = base[p];
    if (f) v += mix * f[p];
    for (int i = 0; i < r; ++i) v -= A[(long)i * lda + p] * cs[i];
    y[p] = v;
  }
}

// per-CTA maxima of the absolute row sums, then the maximum of those
__global__ void __launch_bounds__(MX_NT)
k_absrow_part(const double* __restrict__ A, long lda, int r, long n, double* __restrict__ part) {
  __shared__ double sh[MX_NT / 32];
  double mx = 0.0;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < r; ++i) s += fabs(A[(long)i * lda + p]);
    mx = fmax(mx, s);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < MX_NT / 32; ++w) m = fmax(m, sh[w]);
    part[blockIdx.x] = m;
  }
}

__global__ void k_absrow_final(const double* __restrict__ part, int np, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double m = 0.0;
    for (int i = 0; i < np; ++i) m = fmax(m, part[i]);
    out[0] = m;
  }
}

extern "C" int psc_mix2_diff(psc_ctx* ctx, const double* x1, const double* f1, double* dx, double* df, double mix,
                             void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, x1 && f1 && dx && df, "mix2_diff: NULL pointer");
  k_mix2_diff<<<PSC_RED_BLOCKS, MX_NT, 0, (cudaStream_t)stream>>>(x1, f1, dx, df, mix, ctx->n);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_mix2_store(psc_ctx* ctx, const double* x1, const double* f1, double* dx, double* df,
                              void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, x1 && f1 && dx && df, "mix2_store: NULL pointer");
  k_mix2_store<<<PSC_RED_BLOCKS, MX_NT, 0, (cudaStream_t)stream>>>(x1, f1, dx, df, ctx->n);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_block_dots(psc_ctx* ctx, const double* A, long lda, int r, const double* x, double* out_dev,
                              void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, r >= 0 && (r == 0 || (A && x && out_dev)) && lda >= ctx->n, "block_dots: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  for (int i0 = 0; i0 < r; i0 += PSC_RED_SLOTS) {
    const int ns = std::min(PSC_RED_SLOTS, r - i0);
    const double* a[PSC_RED_SLOTS];
    const double* b[PSC_RED_SLOTS];
    for (int s = 0; s < ns; ++s) {
      a[s] = A + (long)(i0 + s) * lda;
      b[s] = x;
    }
    if (int rc = psc_dots(ctx, ns, a, b, ctx->n, out_dev + i0, st)) return rc;
  }
  return 0;
}

extern "C" int psc_block_combine(psc_ctx* ctx, double* y, const double* base, const double* f, double mix,
                                 const double* A, long lda, int r, const double* c_dev, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, y && base && r >= 0 && (r == 0 || (A && c_dev)) && lda >= ctx->n, "block_combine: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  // chunks of MX_COEF columns; the first carries base and f, later ones
  // continue from y
  int i0 = 0;
  do {
    const int nr = std::min(MX_COEF, r - i0);
    k_block_combine<<<PSC_RED_BLOCKS, MX_NT, 0, st>>>(y, i0 == 0 ? base : y, i0 == 0 ? f : nullptr, mix,
                                                      A ? A + (long)i0 * lda : nullptr, lda, nr,
                                                      c_dev ? c_dev + i0 : nullptr, ctx->n);
    PSC_LAUNCH_CHECK(ctx);
    i0 += nr;
  } while (i0 < r);
  return 0;
}

extern "C" int psc_block_absrow_max(psc_ctx* ctx, const double* A, long lda, int r, double* out_dev, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, A && out_dev && r >= 1 && lda >= ctx->n, "block_absrow_max: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  k_absrow_part<<<PSC_RED_BLOCKS, MX_NT, 0, st>>>(A, lda, r, ctx->n, ctx->red_partial);
  PSC_LAUNCH_CHECK(ctx);
  k_absrow_final<<<1, 32, 0, st>>>(ctx->red_partial, PSC_RED_BLOCKS, out_dev);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}
