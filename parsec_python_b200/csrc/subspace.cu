// Subspace Rayleigh-Ritz without an explicit orthonormal basis.
//
// The reference orthonormalises the filtered block W by Householder QR
// (Eigensolvers/chefsi1.py:43, first_filt.py:43) and then forms
// G = Q^T H Q (chefsi1.py:46-54).  The same Ritz pairs follow from the two
// Gram matrices of W itself:  with  S = W^T W = R^T R  (Cholesky) and
// K = W^T (H W),  the Ritz values are the eigenvalues of  R^{-T} K R^{-1}
// and the Ritz vectors are  W R^{-1} Y.  So one pass over W and HW gives both
// Grams, all k x k work (Cholesky, triangular inverse, two k^3 products, the
// symmetric eigensolver) stays FP64 on the device, and a single block product
// W T, T = R^{-1} Y, replaces the two CholeskyQR passes plus W Q.
//
// Kernels:
//   k_gram_pair  per row chunk, S and K partials (64 x 64 output tile, one
//                8 x 8 register tile per thread, rows staged in shared memory)
//   k_gemm_tall  Out = W T for n x k by k x kout (128 rows x 64 columns per
//                CTA, 4 x 8 register tile per thread)
//   k_small_mm   C = op(A) B for k x k matrices (64 x 64 shared-memory tiles)
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>

namespace {
constexpr int GP_T = 64;   // output tile
constexpr int GP_R = 16;   // rows staged per step
}  // namespace

// threads 0..63 accumulate S = A^T A tile, threads 64..127 K = A^T B tile
template <typename T>
__global__ void __launch_bounds__(128)
k_gram_pair(const T* __restrict__ A, const T* __restrict__ B, long ld, int k, long n, long chunk, int tiles,
            double* __restrict__ partS, double* __restrict__ partK) {
  // column-major tiles [column][row], rows padded by one: staging writes
  // (consecutive rows) and the compute reads (columns 2t + 16m) are both
  // free of bank conflicts
  __shared__ double As[GP_T][GP_R + 1];
  __shared__ double Bsh[GP_T][GP_R + 1];
  __shared__ double At[GP_T][GP_R + 1];
  const int ti = blockIdx.y / tiles, tj = blockIdx.y % tiles;
  const long r0 = (long)blockIdx.x * chunk;
  const long r1 = min(n, r0 + chunk);
  const int which = threadIdx.x >> 6;      // 0: S, 1: K
  const int lt = threadIdx.x & 63;
  // 8 x 8 thread grid; thread (tr, tc) owns rows 2tr + 16m + {0,1} and
  // columns 2tc + 16m + {0,1}, m = 0..3 (interleaved: conflict-free 16-byte loads)
  const int tr = lt >> 3, tc = lt & 7;
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  for (long rb = r0; rb < r1; rb += GP_R) {
    for (int e = threadIdx.x; e < GP_R * GP_T; e += 128) {
      const int r = e % GP_R, c = e / GP_R;
      const long row = rb + r;
      const int ca = ti * GP_T + c, cb = tj * GP_T + c;
      const bool ok = row < r1;
      As[c][r] = (ok && ca < k) ? (double)A[row + (long)ca * ld] : 0.0;
      At[c][r] = (ok && cb < k) ? (double)A[row + (long)cb * ld] : 0.0;
      Bsh[c][r] = (ok && cb < k) ? (double)B[row + (long)cb * ld] : 0.0;
    }
    __syncthreads();
    const double (*R)[GP_R + 1] = which ? Bsh : At;
#pragma unroll 4
    for (int r = 0; r < GP_R; ++r) {
      double a[8], b[8];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        a[2 * m] = As[2 * tr + 16 * m][r];
        a[2 * m + 1] = As[2 * tr + 16 * m + 1][r];
        b[2 * m] = R[2 * tc + 16 * m][r];
        b[2 * m + 1] = R[2 * tc + 16 * m + 1][r];
      }
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
  double* out = (which ? partK : partS) + (long)blockIdx.x * k * k;
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int gi = ti * GP_T + 2 * tr + 16 * (i >> 1) + (i & 1);
      const int gj = tj * GP_T + 2 * tc + 16 * (j >> 1) + (j & 1);
      if (gi < k && gj < k) out[gi + (long)gj * k] = acc[i][j];
    }
}

// sum partials in fixed order, one warp per entry (lanes take every 32nd
// chunk, then a fixed shuffle tree); S symmetrised as 0.5 (S + S^T), K likewise
__global__ void k_gram_pair_final(const double* __restrict__ partS, const double* __restrict__ partK, int nchunk,
                                  int k, double* __restrict__ S, double* __restrict__ K) {
  const long kk = (long)k * k;
  const int lane = threadIdx.x & 31;
  const long nwarps = (long)gridDim.x * (blockDim.x >> 5);
  for (long e = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < 2 * kk; e += nwarps) {
    const bool isK = e >= kk;
    const long f = isK ? e - kk : e;
    const int i = (int)(f % k), j = (int)(f / k);
    const long t = j + (long)i * k;
    const double* P = isK ? partK : partS;
    double s = 0.0, u = 0.0;
    for (int c = lane; c < nchunk; c += 32) {
      s += P[(long)c * kk + f];
      u += P[(long)c * kk + t];
    }
    s = psc_warp_sum(s);
    u = psc_warp_sum(u);
    if (lane == 0) (isK ? K : S)[f] = 0.5 * (s + u);
  }
}

// Out (n x kout) = W (n x k) T (k x kout): 128 rows x 64 columns per CTA,
// thread (tr, tc) owns rows tr + 32a (a = 0..3) and columns 8tc..8tc+7
template <typename T>
__global__ void __launch_bounds__(256)
k_gemm_tall(const T* __restrict__ W, long ldw, int k, const double* __restrict__ Tm, int kout, T* __restrict__ O,
            long ldo, long n) {
  constexpr int BR = 128, BC = 64, KC = 32;
  __shared__ __align__(16) double Ws[KC][BR];
  __shared__ __align__(16) double Ts[KC][BC];
  const long row0 = (long)blockIdx.x * BR;
  const int c0 = blockIdx.y * BC;
  const int tr = threadIdx.x & 31, tc = threadIdx.x >> 5;
  double acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  for (int i0 = 0; i0 < k; i0 += KC) {
    const int ni = min(KC, k - i0);
    for (int e = threadIdx.x; e < KC * BR; e += 256) {
      const int i = e / BR, r = e % BR;
      const long row = row0 + r;
      Ws[i][r] = (i < ni && row < n) ? (double)W[row + (long)(i0 + i) * ldw] : 0.0;
    }
    for (int e = threadIdx.x; e < KC * BC; e += 256) {
      const int i = e / BC, c = e % BC;
      Ts[i][c] = (i < ni && c0 + c < kout) ? Tm[(i0 + i) + (long)(c0 + c) * k] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int i = 0; i < KC; ++i) {
      const double w[4] = {Ws[i][tr], Ws[i][tr + 32], Ws[i][tr + 64], Ws[i][tr + 96]};
      double t[8];
#pragma unroll
      for (int j = 0; j < 8; j += 2) {
        const double2 v = *reinterpret_cast<const double2*>(&Ts[i][8 * tc + j]);
        t[j] = v.x;
        t[j + 1] = v.y;
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] += w[a] * t[b];
    }
    __syncthreads();
  }
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const int c = c0 + 8 * tc + b;
    if (c >= kout) continue;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const long row = row0 + tr + 32 * a;
      if (row < n) O[row + (long)c * ldo] = (T)acc[a][b];
    }
  }
}

// C (k x k) = op(A) B, op = transpose if ta; column-major k x k.  64 x 64
// output tile per CTA, 4 x 4 per thread, the reduction staged 16 at a time
// in shared memory; every output is summed over l in increasing order (the
// order of a plain dot product).
constexpr int SM_T = 64, SM_K = 16;
__global__ void __launch_bounds__(256)
k_small_mm(const double* __restrict__ A, const double* __restrict__ B, int k, int ta, double* __restrict__ C) {
  __shared__ double As[SM_K][SM_T + 1];   // As[l][i] = op(A)[i0 + i, l0 + l]
  __shared__ double Bs[SM_K][SM_T + 1];   // Bs[l][j] = B[l0 + l, j0 + j]
  const int i0 = blockIdx.x * SM_T, j0 = blockIdx.y * SM_T;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // outputs i0 + tx + 16 a, j0 + ty + 16 b
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
  for (int l0 = 0; l0 < k; l0 += SM_K) {
    for (int e = threadIdx.x; e < SM_K * SM_T; e += 256) {
      // A: for ta the reduction index is A's row (contiguous): e -> (l fastest)
      int l, i;
      if (ta) { l = e % SM_K; i = e / SM_K; } else { i = e % SM_T; l = e / SM_T; }
      const int gi = i0 + i, gl = l0 + l;
      As[l][i] = (gi < k && gl < k) ? (ta ? A[gl + (long)gi * k] : A[gi + (long)gl * k]) : 0.0;
      const int bl = e % SM_K, bj = e / SM_K;
      const int gbl = l0 + bl, gj = j0 + bj;
      Bs[bl][bj] = (gbl < k && gj < k) ? B[gbl + (long)gj * k] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int l = 0; l < SM_K; ++l) {
      double av[4], bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = As[l][tx + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) bv[b] = Bs[l][ty + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = i0 + tx + 16 * a, j = j0 + ty + 16 * b;
      if (i < k && j < k) C[i + (long)j * k] = acc[a][b];
    }
}

// dense.cu
int psc_chol_inv_dev(psc_ctx* ctx, double* S, int k, double* X, cudaStream_t st);

int psc_gemm_tall(psc_ctx* ctx, int dtype, const void* W, long ldw, int k, const double* Tm, int kout, void* O,
                  long ldo, cudaStream_t st) {
  PSC_REQUIRE(ctx, W != O, "gemm: output must not alias input");
  if (dtype == PSC_F32) {
    const int rc = psc_gemm_tall_tc(ctx, (const float*)W, ldw, k, Tm, kout, (float*)O, ldo, st);
    if (rc >= 0) return rc;
  }
  dim3 grid(psc_div_up(ctx->n, 128), psc_div_up(kout, 64));
  if (dtype == PSC_F64)
    k_gemm_tall<double><<<grid, 256, 0, st>>>((const double*)W, ldw, k, Tm, kout, (double*)O, ldo, ctx->n);
  else
    k_gemm_tall<float><<<grid, 256, 0, st>>>((const float*)W, ldw, k, Tm, kout, (float*)O, ldo, ctx->n);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

static int gram_pair(psc_ctx* ctx, int dtype, const void* W, const void* V, long ld, int k, double* S, double* K,
                     cudaStream_t st) {
  if (dtype == PSC_F32) {
    const int rc = psc_gram_pair_tc(ctx, (const float*)W, (const float*)V, ld, k, S, K, st);
    if (rc >= 0) return rc;
  }
  const long n = ctx->n;
  const int tiles = (k + GP_T - 1) / GP_T;
  const int ntile = tiles * tiles;
  // two waves of two CTAs per SM (the kernel holds 204 registers per thread)
  int nchunk = std::max(1, std::min(ctx->gram_blocks / 2, (148 * 4 + ntile - 1) / ntile));
  nchunk = (int)std::min<long>(nchunk, std::max<long>(1, n / GP_R));
  const long chunk = ((n + nchunk - 1) / nchunk + GP_R - 1) / GP_R * GP_R;
  nchunk = (int)((n + chunk - 1) / chunk);
  double* partS = ctx->gram_partial;
  double* partK = ctx->gram_partial + (size_t)nchunk * k * k;
  dim3 grid(nchunk, ntile);
  if (dtype == PSC_F64)
    k_gram_pair<double><<<grid, 128, 0, st>>>((const double*)W, (const double*)V, ld, k, n, chunk, tiles, partS,
                                               partK);
  else
    k_gram_pair<float><<<grid, 128, 0, st>>>((const float*)W, (const float*)V, ld, k, n, chunk, tiles, partS,
                                              partK);
  PSC_LAUNCH_CHECK(ctx);
  const long kk = (long)k * k;
  k_gram_pair_final<<<std::max(1, (int)std::min<long>(148 * 8, (2 * kk + 7) / 8)), 256, 0, st>>>(partS, partK,
                                                                                               nchunk, k, S, K);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

// S = W^T W and K = W^T V (k x k, column-major FP64 on the device).
extern "C" int psc_gram_pair(psc_ctx* ctx, int dtype, const void* W, const void* V, long ld, int k, double* S,
                             double* K, void* stream) {
  if (!ctx) return 2;
  if (psc_ensure_dense(ctx, k)) return 1;
  PSC_REQUIRE(ctx, W && V && S && K && ld >= ctx->n, "gram_pair: bad arguments");
  return gram_pair(ctx, dtype, W, V, ld, k, S, K, (cudaStream_t)stream);
}

// Rayleigh-Ritz of the (not necessarily orthonormal) block W: V = H W,
// S = W^T W, K = W^T V, S = R^T R, M = R^{-T} K R^{-1} = Y diag(ritz) Y^T,
// result W R^{-1} Y written to V.  ritz ascending.
extern "C" int psc_subspace_rr(psc_ctx* ctx, int dtype, const void* W, void* V, long ld, int k, double* ritz_dev,
                               void* stream) {
  if (!ctx) return 2;
  cudaStream_t st = (cudaStream_t)stream;
  if (psc_ensure_dense(ctx, k)) return 1;
  PSC_REQUIRE(ctx, W != V && ld >= ctx->n, "subspace_rr: bad arguments");
  int rc = psc_apply_h_impl(ctx, dtype, W, ld, V, ld, nullptr, 0, k, nullptr, 1.0, 0.0, 0.0, st);
  if (rc) return rc;
  double* S = ctx->gram;    // -> R
  double* K = ctx->gram2;   // -> scratch
  double* Ri = ctx->tri;    // R^{-1}
  double* Y = ctx->evec;
  rc = gram_pair(ctx, dtype, W, V, ld, k, S, K, st);
  if (rc) return rc;
  rc = psc_chol_inv_dev(ctx, S, k, Ri, st);
  if (rc) return rc;
  const dim3 gmm(psc_div_up(k, SM_T), psc_div_up(k, SM_T));
  // S <- K R^{-1}; K <- R^{-T} S  (M, symmetric up to rounding)
  k_small_mm<<<gmm, 256, 0, st>>>(K, Ri, k, 0, S);
  PSC_LAUNCH_CHECK(ctx);
  k_small_mm<<<gmm, 256, 0, st>>>(Ri, S, k, 1, K);
  PSC_LAUNCH_CHECK(ctx);
  rc = psc_syev_impl(ctx, K, k, ritz_dev, Y, st);
  if (rc) return rc;
  // S <- R^{-1} Y
  k_small_mm<<<gmm, 256, 0, st>>>(Ri, Y, k, 0, S);
  PSC_LAUNCH_CHECK(ctx);
  return psc_gemm_tall(ctx, dtype, W, ld, k, S, k, V, ld, st);
}
