// Subspace linear algebra: Gram products W^T V (n x k -> k x k), block
// products W*Q, Cholesky, triangular inverse and a one-CTA cyclic Jacobi
// symmetric eigensolver, plus the two subspace drivers built from them:
// CholeskyQR2 orthonormalisation (replaces the Householder QR at
// Eigensolvers/chefsi1.py:43 and first_filt.py:43) and Rayleigh-Ritz
// (chefsi1.py:46-67, first_filt.py:44-63).  Small k x k work is FP64.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>
#include <cmath>

// ---------------------------------------------------------------------------
// Gram partials: partial[chunk] (k1 x k2, column-major) = A[rows]^T B[rows]
// ---------------------------------------------------------------------------
constexpr int GT = 64;  // output tile edge
constexpr int GR = 32;  // rows staged per step

template <typename T>
__global__ void __launch_bounds__(256)
k_gram_partial(const T* __restrict__ A, long lda, int k1, const T* __restrict__ B, long ldb, int k2, long n,
               long chunk, int tiles_j, int upper_only, double* __restrict__ partial) {
  __shared__ double As[GR][GT + 1];
  __shared__ double Bs[GR][GT + 1];
  const int ti = blockIdx.y / tiles_j, tj = blockIdx.y % tiles_j;
  if (upper_only && ti > tj) return;
  const long r0 = (long)blockIdx.x * chunk;
  const long r1 = min(n, r0 + chunk);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (long rb = r0; rb < r1; rb += GR) {
    for (int e = threadIdx.x; e < GR * GT; e += 256) {
      const int r = e % GR, c = e / GR;
      const long row = rb + r;
      const int ca = ti * GT + c, cb = tj * GT + c;
      As[r][c] = (row < r1 && ca < k1) ? (double)A[row + (long)ca * lda] : 0.0;
      Bs[r][c] = (row < r1 && cb < k2) ? (double)B[row + (long)cb * ldb] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int r = 0; r < GR; ++r) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[r][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[r][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
  double* out = partial + (long)blockIdx.x * k1 * k2;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gi = ti * GT + ty + 16 * i, gj = tj * GT + tx + 16 * j;
      if (gi < k1 && gj < k2) out[gi + (long)gj * k1] = acc[i][j];
    }
}

// out = sum over chunks (fixed order); mode 0: plain, 1: mirror the upper
// triangle (G[i,j] = M[i,j] for i <= j, as the reference's dot loop), 2: 0.5(M+M^T)
__global__ void k_gram_final(const double* __restrict__ partial, int nchunk, int k1, int k2, int mode,
                             double* __restrict__ out) {
  const long kk = (long)k1 * k2;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < kk; e += (long)gridDim.x * blockDim.x) {
    const int i = (int)(e % k1), j = (int)(e / k1);
    long src = e;
    if (mode == 1 && i > j) src = j + (long)i * k1;
    double s = 0.0;
    for (int c = 0; c < nchunk; ++c) s += partial[(long)c * kk + src];
    if (mode == 2) {
      double t = 0.0;
      const long tr = j + (long)i * k1;
      for (int c = 0; c < nchunk; ++c) t += partial[(long)c * kk + tr];
      s = 0.5 * (s + t);
    }
    out[e] = s;
  }
}

int psc_ensure_dense(psc_ctx* ctx, int k) {
  PSC_REQUIRE(ctx, k >= 1 && k <= PSC_MAX_K, "subspace width out of range");
  if (k <= ctx->dense_cap) return 0;
  psc_dfree(ctx->gram); psc_dfree(ctx->gram2); psc_dfree(ctx->evec); psc_dfree(ctx->tri); psc_dfree(ctx->gram_partial);
  psc_dfree(ctx->jac_v);
  const int cap = std::max(k, 64);
  const size_t kk = (size_t)cap * cap;
  // Jacobi scratch: padded A and V of order <= cap + 1 when they do not fit on chip
  PSC_CUDA(ctx, psc_dmalloc(&ctx->jac_v, 2 * (size_t)(cap + 2) * (cap + 2) * sizeof(double)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->gram, kk * sizeof(double)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->gram2, kk * sizeof(double)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->evec, kk * sizeof(double)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->tri, kk * sizeof(double)));
  // per-chunk partial k x k tiles: enough chunks for two waves of two CTAs per
  // SM at small k, at most 128 MB of partials at large k
  ctx->gram_blocks = std::min(1184, std::max(296, (int)(16777216 / (long)kk)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->gram_partial, (size_t)ctx->gram_blocks * kk * sizeof(double)));
  ctx->dense_cap = cap;
  return 0;
}

int psc_gram_impl(psc_ctx* ctx, int dtype, const void* A, long lda, const void* B, long ldb, int k, double* out,
                  int mode, cudaStream_t st) {
  if (psc_ensure_dense(ctx, k)) return 1;
  const long n = ctx->n;
  const int tiles = (k + GT - 1) / GT;
  const int ntile = tiles * tiles;
  int nchunk = std::max(1, std::min(ctx->gram_blocks, (148 * 4 + ntile - 1) / ntile));
  nchunk = (int)std::min<long>(nchunk, std::max<long>(1, n / GR));
  const long chunk = ((n + nchunk - 1) / nchunk + GR - 1) / GR * GR;
  nchunk = (int)((n + chunk - 1) / chunk);
  dim3 grid(nchunk, ntile);
  const int upper = (mode == 1) ? 1 : 0;
  if (dtype == PSC_F64)
    k_gram_partial<double><<<grid, 256, 0, st>>>((const double*)A, lda, k, (const double*)B, ldb, k, n, chunk,
                                                  tiles, upper, ctx->gram_partial);
  else
    k_gram_partial<float><<<grid, 256, 0, st>>>((const float*)A, lda, k, (const float*)B, ldb, k, n, chunk, tiles,
                                                 upper, ctx->gram_partial);
  PSC_LAUNCH_CHECK(ctx);
  const long kk = (long)k * k;
  k_gram_final<<<std::max(1, (int)std::min<long>(592, (kk + 255) / 256)), 256, 0, st>>>(ctx->gram_partial, nchunk, k,
                                                                                    k, mode, out);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_gram(psc_ctx* ctx, int dtype, const void* A, long lda, const void* B, long ldb, int k,
                        int mode, double* out_dev, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, lda >= ctx->n && ldb >= ctx->n, "gram: ld < n");
  return psc_gram_impl(ctx, dtype, A, lda, B, ldb, k, out_dev, mode, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Out (n x kout) = W (n x k) * Q (k x kout, FP64, column-major): k_gemm_tall
// in subspace.cu
// ---------------------------------------------------------------------------
int psc_gemm_tall(psc_ctx* ctx, int dtype, const void* W, long ldw, int k, const double* Tm, int kout, void* O,
                  long ldo, cudaStream_t st);

int psc_gemm_nn_impl(psc_ctx* ctx, int dtype, const void* W, long ldw, int k, const double* Q, int kout, void* out,
                     long ldo, cudaStream_t st) {
  return psc_gemm_tall(ctx, dtype, W, ldw, k, Q, kout, out, ldo, st);
}

extern "C" int psc_gemm_nn(psc_ctx* ctx, int dtype, const void* W, long ldw, int k, const double* Q, int kout,
                           void* out, long ldo, void* stream) {
  if (!ctx) return 2;
  return psc_gemm_nn_impl(ctx, dtype, W, ldw, k, Q, kout, out, ldo, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Cholesky (upper, G = R^T R, in place, one CTA) and upper-triangular inverse
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_cholesky(double* A, int k, int* status) {
  for (int j = 0; j < k; ++j) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const double d = A[j + (long)j * k];
      if (!(d > 0.0)) status[1] = j + 1;  // not positive definite
      A[j + (long)j * k] = d > 0.0 ? sqrt(d) : 1.0;
    }
    __syncthreads();
    const double rjj = A[j + (long)j * k];
    for (int c = j + 1 + threadIdx.x; c < k; c += blockDim.x) A[j + (long)c * k] /= rjj;
    __syncthreads();
    const int m = k - j - 1;
    for (long e = threadIdx.x; e < (long)m * m; e += blockDim.x) {
      const int r = j + 1 + (int)(e % m), c = j + 1 + (int)(e / m);
      if (r <= c) A[r + (long)c * k] -= A[j + (long)r * k] * A[j + (long)c * k];
    }
  }
  __syncthreads();
  for (long e = threadIdx.x; e < (long)k * k; e += blockDim.x) {
    const int r = (int)(e % k), c = (int)(e / k);
    if (r > c) A[e] = 0.0;
  }
}

__global__ void k_triu_inv(const double* __restrict__ R, int k, double* __restrict__ X) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x) {
    double* xj = X + (long)j * k;
    for (int i = j + 1; i < k; ++i) xj[i] = 0.0;
    xj[j] = 1.0 / R[j + (long)j * k];
    for (int i = j - 1; i >= 0; --i) {
      double s = 0.0;
      for (int l = i + 1; l <= j; ++l) s += R[i + (long)l * k] * xj[l];
      xj[i] = -s / R[i + (long)i * k];
    }
  }
}

// ---------------------------------------------------------------------------
// Cyclic Jacobi eigensolver, one CTA.  The matrix is padded to even order m
// (a zero row/column when k is odd) and symmetrised.  Each round of a sweep
// pairs the m indices into m/2 disjoint planes (circle method); the round is
// two steps separated by one barrier each:
//   1. every plane computes its rotation or skips it while
//      |a_pq| <= 1e-17 (|a_pp| + |a_qq|).  The angle comes from FP32
//      arithmetic (short latency); c and s are normalised in FP64, so every
//      rotation is orthogonal to FP64 rounding and the a_pq it leaves
//      (~1e-7 of the old one) is annihilated by later sweeps;
//   2. the two-sided update A <- P^T A P as independent 2x2 blocks (rows of
//      plane i, columns of plane j) on a 32-wide thread grid, together with
//      V <- V P.
// The solver has converged when a whole sweep rotates nothing (at most 60
// sweeps; status word 2 is set otherwise).  Eigenvalues ascending,
// eigenvectors permuted to match.
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(NT)
k_jacobi(const double* __restrict__ Ain, int k, double* __restrict__ evals, double* __restrict__ Vout,
         int use_smem, double* __restrict__ scratch, int* status) {
  extern __shared__ double sm[];
  __shared__ int rp[512], rq[512];
  __shared__ double rc[512], rs[512];
  __shared__ int rank_of[1024];
  __shared__ int nrot;
  const int m = k + (k & 1);
  const int half = m / 2;
  const int ld = m + 1;   // odd leading dimension: a warp's strided accesses spread over the banks
  // use_smem: 2 = A and V on chip, 1 = A on chip and V in global scratch, 0 = both in scratch
  double* A = use_smem ? sm : scratch;
  double* V = use_smem == 2 ? A + m * ld : scratch + (use_smem ? 0 : m * ld);
  for (int e = threadIdx.x; e < m * m; e += NT) {
    const int i = e % m, j = e / m;
    double a = 0.0;
    if (i < k && j < k) a = (i == j) ? Ain[i + j * k] : 0.5 * (Ain[i + j * k] + Ain[j + i * k]);
    A[i + j * ld] = a;
    V[i + j * ld] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  int sweeps_done = 0;
  for (int sweep = 0; sweep < 60 && k > 1; ++sweep) {
    sweeps_done = sweep + 1;
    if (threadIdx.x == 0) nrot = 0;
    __syncthreads();
    for (int r = 0; r < m - 1; ++r) {
      for (int i = threadIdx.x; i < half; i += NT) {
        const int a = (i == 0) ? 0 : ((i - 1 + r) % (m - 1)) + 1;
        const int b = ((m - 2 - i + r) % (m - 1)) + 1;
        const int p = min(a, b), q = max(a, b);
        double c = 1.0, s = 0.0;
        const double apq = A[p + q * ld];
        const double app = A[p + p * ld], aqq = A[q + q * ld];
        if (apq != 0.0 && fabs(apq) > 1e-17 * (fabs(app) + fabs(aqq))) {
          nrot = 1;   // benign: every writer stores the same value
          s = 1.0;
          const double theta = (aqq - app) / (2.0 * apq);
          double t;
          if (fabs(theta) > 1e18) {
            t = 0.5 / theta;
          } else {
            // tan of the annihilating angle to FP32 accuracy (Rutishauser's
            // form); the rotation stays exactly orthogonal below, and the
            // remainder of a_pq is removed by later sweeps
            const float th = (float)theta;
            t = (double)(copysignf(1.0f, th) / (fabsf(th) + sqrtf(fmaf(th, th, 1.0f))));
          }
          // c = 1/sqrt(1+t^2) in FP64: FP32 estimate plus two Newton-Raphson
          // steps y <- y (3 - x y^2) / 2
          const double x = fma(t, t, 1.0);
          double y = (double)rsqrtf((float)x);
          y = y * (1.5 - 0.5 * x * y * y);
          y = y * (1.5 - 0.5 * x * y * y);
          c = y;
          s = t * y;
        }
        rp[i] = p; rq[i] = q; rc[i] = c; rs[i] = s;
      }
      __syncthreads();
      // 2x2 blocks (i, j) on a 32-wide thread grid, then the V columns
      {
        const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
        for (int i = ty; i < half; i += NT / 32) {
          const double si = rs[i];
          const int pi = rp[i], qi = rq[i];
          const double ci = rc[i];
          for (int j = tx; j < half; j += 32) {
            const double sj = rs[j];
            if (si == 0.0 && sj == 0.0) continue;
            const int pj = rp[j], qj = rq[j];
            const double cj = rc[j];
            const double x00 = A[pi + pj * ld], x01 = A[pi + qj * ld], x10 = A[qi + pj * ld], x11 = A[qi + qj * ld];
            // columns (plane j): [x.0 x.1] <- [c x.0 - s x.1, s x.0 + c x.1]
            const double y00 = cj * x00 - sj * x01, y01 = sj * x00 + cj * x01;
            const double y10 = cj * x10 - sj * x11, y11 = sj * x10 + cj * x11;
            // rows (plane i); the rotated pair's own block is kept exactly symmetric
            const double z00 = ci * y00 - si * y10, z10 = si * y00 + ci * y10;
            const double z01 = ci * y01 - si * y11, z11 = si * y01 + ci * y11;
            if (i == j) {
              const double off = 0.5 * (z01 + z10);
              A[pi + pj * ld] = z00;
              A[qi + qj * ld] = z11;
              A[qi + pj * ld] = off;
              A[pi + qj * ld] = off;
            } else {
              A[pi + pj * ld] = z00;
              A[qi + pj * ld] = z10;
              A[pi + qj * ld] = z01;
              A[qi + qj * ld] = z11;
            }
          }
        }
        for (int j = ty; j < half; j += NT / 32) {
          const double sj = rs[j];
          if (sj == 0.0) continue;
          const double cj = rc[j];
          double* vp = V + rp[j] * ld;
          double* vq = V + rq[j] * ld;
          for (int row = tx; row < m; row += 32) {
            const double x = vp[row], y = vq[row];
            vp[row] = cj * x - sj * y;
            vq[row] = sj * x + cj * y;
          }
        }
      }
      __syncthreads();
    }
    // a sweep without rotations means every pair is diagonal to working precision
    const int rotated = nrot;
    __syncthreads();
    if (rotated == 0) break;
    if (threadIdx.x == 0 && sweep == 59) status[2] = 1;  // did not converge
  }
  if (threadIdx.x == 0) status[6] = sweeps_done;   // diagnostic: sweeps of the last solve
  __syncthreads();
  // sort ascending (stable by index), then permute the eigenvectors with
  // coalesced stores
  for (int i = threadIdx.x; i < k; i += NT) {
    const double li = A[i + i * ld];
    int rank = 0;
    for (int j = 0; j < k; ++j) {
      const double lj = A[j + j * ld];
      rank += (lj < li) || (lj == li && j < i);
    }
    evals[rank] = li;
    rank_of[rank] = i;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < k * k; e += NT) {
    const int col = e / k, r = e - col * k;
    Vout[e] = V[r + rank_of[col] * ld];
  }
}

int psc_syev_impl(psc_ctx* ctx, double* A, int k, double* evals, double* evecs, cudaStream_t st) {
  PSC_REQUIRE(ctx, k >= 1 && k <= 1022, "syev: k out of range");
  if (psc_ensure_dense(ctx, k)) return 1;
  const int m = k + (k & 1);
  const size_t tile = (size_t)m * (m + 1) * sizeof(double);
  const int use_smem = 2 * tile <= 200 * 1024 ? 2 : (tile <= 200 * 1024 ? 1 : 0);
  const size_t dyn = use_smem * tile;
  // CTA size matched to the (m/2)^2 blocks + (m/2) m rows of a rotation round
#define PSC_JACOBI(NTH)                                                                                   \
  {                                                                                                       \
    if (use_smem)                                                                                         \
      PSC_CUDA(ctx, cudaFuncSetAttribute(k_jacobi<NTH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn)); \
    k_jacobi<NTH><<<1, NTH, dyn, st>>>(A, k, evals, evecs, use_smem, ctx->jac_v, ctx->dev_status);       \
  }
  // 32 x (NT/32) thread grid over the (m/2)^2 blocks of a rotation round
  const int half = m / 2;
  if (half <= 8) PSC_JACOBI(256)
  else if (half <= 16) PSC_JACOBI(512)
  else PSC_JACOBI(1024)
#undef PSC_JACOBI
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_syev(psc_ctx* ctx, double* A, int k, double* evals, double* evecs, void* stream) {
  if (!ctx) return 2;
  return psc_syev_impl(ctx, A, k, evals, evecs, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// subspace drivers
// ---------------------------------------------------------------------------
// CholeskyQR applied `passes` times: W <- W R^{-1} with W^T W = R^T R.  Uses
// T (same shape) as the second buffer; *which = 0 if the result is in W.
extern "C" int psc_orthonormalize(psc_ctx* ctx, int dtype, void* W, void* T, long ld, int k, int passes,
                                  int* which, void* stream) {
  if (!ctx) return 2;
  cudaStream_t st = (cudaStream_t)stream;
  if (psc_ensure_dense(ctx, k)) return 1;
  void* buf[2] = {W, T};
  int cur = 0;
  for (int p = 0; p < passes; ++p) {
    int rc = psc_gram_impl(ctx, dtype, buf[cur], ld, buf[cur], ld, k, ctx->gram, 2, st);
    if (rc) return rc;
    k_cholesky<<<1, 1024, 0, st>>>(ctx->gram, k, ctx->dev_status);
    PSC_LAUNCH_CHECK(ctx);
    k_triu_inv<<<psc_div_up(k, 128), 128, 0, st>>>(ctx->gram, k, ctx->tri);
    PSC_LAUNCH_CHECK(ctx);
    rc = psc_gemm_nn_impl(ctx, dtype, buf[cur], ld, k, ctx->tri, k, buf[cur ^ 1], ld, st);
    if (rc) return rc;
    cur ^= 1;
  }
  if (which) *which = cur;
  return 0;
}

// Rayleigh-Ritz on an orthonormal W: V = H W, G = W^T H W (upper triangle
// mirrored, as the reference's dot loop), G = Q diag(ritz) Q^T, result W Q is
// written to V.  ritz_dev receives the k Ritz values in ascending order.
extern "C" int psc_rayleigh_ritz(psc_ctx* ctx, int dtype, const void* W, void* V, long ld, int k, double* ritz_dev,
                                 void* stream) {
  if (!ctx) return 2;
  cudaStream_t st = (cudaStream_t)stream;
  if (psc_ensure_dense(ctx, k)) return 1;
  int rc = psc_apply_h_impl(ctx, dtype, W, ld, V, ld, nullptr, 0, k, nullptr, 1.0, 0.0, 0.0, st);
  if (rc) return rc;
  rc = psc_gram_impl(ctx, dtype, V, ld, W, ld, k, ctx->gram, 1, st);
  if (rc) return rc;
  rc = psc_syev_impl(ctx, ctx->gram, k, ritz_dev, ctx->evec, st);
  if (rc) return rc;
  return psc_gemm_nn_impl(ctx, dtype, W, ld, k, ctx->evec, k, V, ld, st);
}

int psc_cholesky_dev(psc_ctx* ctx, double* A, int k, cudaStream_t st) {
  k_cholesky<<<1, 1024, 0, st>>>(A, k, ctx->dev_status);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

int psc_triu_inv_dev(psc_ctx* ctx, const double* R, int k, double* X, cudaStream_t st) {
  k_triu_inv<<<psc_div_up(k, 128), 128, 0, st>>>(R, k, X);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}
