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
// Kernels: the Gram pair and the block product W T run on the FP64 tensor
// cores (dmma.cu) for FP64 blocks, and for FP32 blocks when the tcgen05
// split-TF32 path is off (gram_tc.cu, gemm_tc.cu);
//   k_small_mm   C = op(A) B for k x k matrices (64 x 64 shared-memory tiles)
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>

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
  return psc_gemm_tall_dmma(ctx, dtype, W, ldw, k, Tm, kout, O, ldo, st);
}

static int gram_pair(psc_ctx* ctx, int dtype, const void* W, const void* V, long ld, int k, double* S, double* K,
                     cudaStream_t st) {
  if (dtype == PSC_F32) {
    const int rc = psc_gram_pair_tc(ctx, (const float*)W, (const float*)V, ld, k, S, K, st);
    if (rc >= 0) return rc;
  }
  return psc_gram_pair_dmma(ctx, dtype, W, V, ld, k, S, K, st);
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
