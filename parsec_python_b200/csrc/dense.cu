// Subspace linear algebra: Gram products W^T V (n x k -> k x k), block
// products W*Q, Cholesky, triangular inverse and a symmetric eigensolver
// (Householder tridiagonalisation, bisection, inverse iteration), plus the
// two subspace drivers built from them:
// CholeskyQR2 orthonormalisation (replaces the Householder QR at
// Eigensolvers/chefsi1.py:43 and first_filt.py:43) and Rayleigh-Ritz
// (chefsi1.py:46-67, first_filt.py:44-63).  Small k x k work is FP64.
#include "psc_internal.cuh"
#include <cooperative_groups.h>
#include "../../include/psc.h"

#include <algorithm>

namespace cg = cooperative_groups;
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
  psc_dfree(ctx->eig_work);
  const int cap = std::max(k, 64);
  const size_t kk = (size_t)cap * cap;
  // eigensolver scratch: reflectors, tridiagonal eigenvectors, T and tau (>= 2 k^2 + 3 k)
  PSC_CUDA(ctx, psc_dmalloc(&ctx->eig_work, 2 * (size_t)(cap + 2) * (cap + 2) * sizeof(double)));
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
// Out (n x kout) = W (n x k) * Q (k x kout, FP64, column-major): subspace.cu
// (tcgen05 or DMMA)
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
// Cholesky S = R^T R (upper R) and R^{-1}
// ---------------------------------------------------------------------------
// Cholesky and inverse in one CTA with the matrix in shared memory (k up to
// 150): S = R^T R (R upper, written back in place with zeros below) and
// X = R^{-1}.
//   column j: every thread reads d = S[j,j] and takes r_jj = sqrt(d) (1, and
//   status word 1 = j + 1, if d <= 0); row j right of the diagonal divided by
//   r_jj goes to u; barrier; the trailing upper triangle loses u_r u_c;
//   barrier.  Two barriers per column.
//   R^{-1}: one warp per column j, right-looking substitution on b = e_j:
//   x_i = b_i / r_ii, then b_r -= R[r, i] x_i for r < i.
constexpr int CI_NT = 512;

static size_t chol_inv_smem_doubles(int k) { return (size_t)k * k + (size_t)(2 + CI_NT / 32) * k; }

__global__ void __launch_bounds__(CI_NT) k_chol_inv(double* __restrict__ S, int k, double* __restrict__ X,
                                                    int* status) {
  extern __shared__ double sm[];
  constexpr int NW = CI_NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  double* A = sm;
  double* u = A + (size_t)k * k;
  double* dg = u + k;
  double* b = dg + k + (size_t)w * k;   // this warp's right-hand side
  for (int c = w; c < k; c += NW)
    for (int r = lane; r < k; r += 32) A[r + (long)c * k] = S[r + (long)c * k];
  __syncthreads();
  for (int j = 0; j < k; ++j) {
    const double d = A[j + (long)j * k];
    const double rjj = d > 0.0 ? sqrt(d) : 1.0;
    if (tid == 0) {
      dg[j] = rjj;
      if (!(d > 0.0)) status[1] = j + 1;   // not positive definite
    }
    for (int c = j + 1 + tid; c < k; c += CI_NT) {
      const double v = A[j + (long)c * k] / rjj;
      u[c] = v;
      A[j + (long)c * k] = v;
    }
    __syncthreads();
    for (int c = j + 1 + w; c < k; c += NW) {
      const double uc = u[c];
      for (int r = j + 1 + lane; r <= c; r += 32) A[r + (long)c * k] -= u[r] * uc;
    }
    __syncthreads();
  }
  for (int c = w; c < k; c += NW)
    for (int r = lane; r < k; r += 32) S[r + (long)c * k] = r < c ? A[r + (long)c * k] : (r == c ? dg[c] : 0.0);
  for (int j = w; j < k; j += NW) {
    double* xj = X + (long)j * k;
    for (int r = lane; r < k; r += 32) {
      if (r <= j) b[r] = r == j ? 1.0 : 0.0;
      else xj[r] = 0.0;
    }
    __syncwarp();
    for (int i = j; i >= 0; --i) {
      const double xi = b[i] / dg[i];
      const double* ri = A + (long)i * k;   // column i of R above the diagonal
      for (int r = lane; r < i; r += 32) b[r] -= ri[r] * xi;
      if (lane == 0) xj[i] = xi;
      __syncwarp();
    }
  }
}

// Blocked right-looking Cholesky for matrices that do not fit one CTA's
// shared memory (k > 151): block columns of CB.  Per block step j0:
//   k_potrf_diag    one CTA factors the CB x CB diagonal block in shared
//                   memory (the k_chol_inv column loop) and writes R11 and
//                   R11^{-T} (the latter into scratch D);
//   k_potrf_panel   R12 = R11^{-T} A12, 64 columns per CTA;
//   k_potrf_update  A22 -= R12^T R12 on the upper triangle, 64 x 64 tiles.
// Then k_trtri_warp forms R^{-1}: one warp per column, the right-looking
// substitution of k_chol_inv with R read from global memory (L2-resident).
constexpr int CB = 64;

__global__ void __launch_bounds__(256) k_potrf_diag(double* __restrict__ A, int k, int j0, double* __restrict__ D,
                                                    int* status) {
  __shared__ double a[CB][CB + 1];   // a[c][r] = A[j0 + r, j0 + c]
  __shared__ double u[CB], dg[CB], dgi[CB];   // dgi = 1 / dg
  const int nb = min(CB, k - j0);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int e = tid; e < nb * nb; e += 256) {
    const int r = e % nb, c = e / nb;
    a[c][r] = A[(j0 + r) + (long)(j0 + c) * k];
  }
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    const double d = a[j][j];
    const double rjj = d > 0.0 ? sqrt(d) : 1.0;
    const double rinv = 1.0 / rjj;
    if (tid == 0) {
      dg[j] = rjj;
      dgi[j] = rinv;
      if (!(d > 0.0) && status[1] == 0) status[1] = j0 + j + 1;   // not positive definite
    }
    for (int c = j + 1 + tid; c < nb; c += 256) {
      const double v = a[c][j] * rinv;
      u[c] = v;
      a[c][j] = v;
    }
    __syncthreads();
    for (int c = j + 1 + w; c < nb; c += 8) {
      const double uc = u[c];
      for (int r = j + 1 + lane; r <= c; r += 32) a[c][r] -= u[r] * uc;
    }
    __syncthreads();
  }
  for (int e = tid; e < nb * nb; e += 256) {
    const int r = e % nb, c = e / nb;
    A[(j0 + r) + (long)(j0 + c) * k] = r < c ? a[c][r] : (r == c ? dg[c] : 0.0);
  }
  // D = R11^{-T} (lower triangular, column-major nb x nb): column j of R11^{-1}
  // by right-looking substitution, one warp per column, stored transposed
  __shared__ double b[8][CB];
  for (int j = w; j < nb; j += 8) {
    for (int r = lane; r < nb; r += 32) b[w][r] = r == j ? 1.0 : 0.0;
    __syncwarp();
    for (int i = j; i >= 0; --i) {
      const double xi = b[w][i] * dgi[i];
      for (int r = lane; r < i; r += 32) b[w][r] -= a[i][r] * xi;
      if (lane == 0) b[w][i] = xi;
      __syncwarp();
    }
    for (int r = lane; r < nb; r += 32) D[j + (long)r * CB] = r <= j ? b[w][r] : 0.0;   // D[j, r] = Rinv[r, j]
    __syncwarp();
  }
}

// R12 (rows j0..j0+nb, columns c >= j0+nb) = D A12 with D = R11^{-T}
__global__ void __launch_bounds__(256) k_potrf_panel(double* __restrict__ A, int k, int j0,
                                                     const double* __restrict__ D) {
  extern __shared__ double psm[];
  double (*d)[CB + 1] = reinterpret_cast<double (*)[CB + 1]>(psm);               // d[l][i] = D[i, l]
  double (*x)[CB + 1] = reinterpret_cast<double (*)[CB + 1]>(psm + CB * (CB + 1));  // 64 columns of A12
  const int nb = min(CB, k - j0);
  const int c0 = j0 + nb + blockIdx.x * 64;
  const int nc = min(64, k - c0);
  for (int e = threadIdx.x; e < nb * nb; e += 256) d[e / nb][e % nb] = D[(e % nb) + (long)(e / nb) * CB];
  for (int e = threadIdx.x; e < nb * nc; e += 256) {
    const int r = e % nb, c = e / nb;
    x[c][r] = A[(j0 + r) + (long)(c0 + c) * k];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nb * nc; e += 256) {
    const int i = e % nb, c = e / nb;
    double s = 0.0;
    for (int l = 0; l <= i; ++l) s += d[l][i] * x[c][l];
    A[(j0 + i) + (long)(c0 + c) * k] = s;
  }
}

// A22[r, c] -= sum_l R12[l, r] R12[l, c] for j0+nb <= r <= c (upper triangle)
__global__ void __launch_bounds__(256) k_potrf_update(double* __restrict__ A, int k, int j0) {
  const int nb = min(CB, k - j0);
  const int b0 = j0 + nb;
  const int tr = blockIdx.x, tc = blockIdx.y;
  if (tr > tc) return;
  extern __shared__ double usm[];
  double (*pr)[64 + 1] = reinterpret_cast<double (*)[64 + 1]>(usm);                // pr[l][i] = R12[l, r0 + i]
  double (*pc)[64 + 1] = reinterpret_cast<double (*)[64 + 1]>(usm + CB * (64 + 1));
  const int r0 = b0 + tr * 64, cc0 = b0 + tc * 64;
  for (int e = threadIdx.x; e < nb * 64; e += 256) {
    const int l = e % nb, i = e / nb;
    pr[l][i] = (r0 + i < k) ? A[(j0 + l) + (long)(r0 + i) * k] : 0.0;
    pc[l][i] = (cc0 + i < k) ? A[(j0 + l) + (long)(cc0 + i) * k] : 0.0;
  }
  __syncthreads();
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[a][q] = 0.0;
  for (int l = 0; l < nb; ++l) {
    double ra[4], cq[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) ra[a] = pr[l][tx + 16 * a];
#pragma unroll
    for (int q = 0; q < 4; ++q) cq[q] = pc[l][ty + 16 * q];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[a][q] += ra[a] * cq[q];
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = r0 + tx + 16 * a, c = cc0 + ty + 16 * q;
      if (r < k && c < k && r <= c) A[r + (long)c * k] -= acc[a][q];
    }
}

__global__ void k_tril_zero(double* A, int k) {
  const long kk = (long)k * k;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < kk; e += (long)gridDim.x * blockDim.x)
    if ((int)(e % k) > (int)(e / k)) A[e] = 0.0;
}

// X = R^{-1}, one warp per column j (8 per CTA): b = e_j, then for i = j .. 0:
// x_i = b_i / r_ii, b_r -= R[r, i] x_i (r < i).  Every step depends on the
// one before, so R's columns are not read from global memory inside the
// steps: the CTA stages the columns it needs (i <= its largest j) in shared
// memory, `ch` at a time from the highest down, rows 0..i of each, with the
// reciprocals of their diagonals.
__global__ void __launch_bounds__(256) k_trtri_warp(const double* __restrict__ R, int k, int ch,
                                                    double* __restrict__ X) {
  extern __shared__ double bs[];   // [8][k] b vectors, [ch][k] staged columns, [ch] 1 / r_ii
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int j = blockIdx.x * 8 + w;
  const int jmax = min(k - 1, blockIdx.x * 8 + 7);
  double* b = bs + (long)w * k;
  double* rs = bs + 8L * k;
  double* rinv = rs + (long)ch * k;
  double* xj = X + (long)j * k;
  if (j < k)
    for (int r = lane; r < k; r += 32) {
      if (r <= j) b[r] = r == j ? 1.0 : 0.0;
      else xj[r] = 0.0;
    }
  for (int c_hi = jmax; c_hi >= 0; c_hi -= ch) {
    const int c_lo = max(0, c_hi - ch + 1);
    const int nr = c_hi + 1;   // rows 0..c_hi cover every staged column's rows 0..i
    __syncthreads();           // the previous chunk has been used by every warp
    for (int e = tid; e < (c_hi - c_lo + 1) * nr; e += 256) {
      const int cc = e / nr, r = e % nr, c = c_lo + cc;
      if (r < c) rs[(long)cc * k + r] = R[r + (long)c * k];
      else if (r == c) rinv[cc] = 1.0 / R[c + (long)c * k];
    }
    __syncthreads();
    if (j < k) {
      for (int i = min(j, c_hi); i >= c_lo; --i) {
        const double* ri = rs + (long)(i - c_lo) * k;
        const double xi = b[i] * rinv[i - c_lo];
        for (int r = lane; r < i; r += 32) b[r] -= ri[r] * xi;
        if (lane == 0) xj[i] = xi;
        __syncwarp();
      }
    }
  }
}

// R and R^{-1} of S = R^T R (S overwritten by R)
int psc_chol_inv_dev(psc_ctx* ctx, double* S, int k, double* X, cudaStream_t st) {
  const size_t dyn = chol_inv_smem_doubles(k) * sizeof(double);
  if (dyn <= 200 * 1024) {
    if (dyn > 48 * 1024)
      PSC_CUDA(ctx, cudaFuncSetAttribute(k_chol_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    k_chol_inv<<<1, CI_NT, dyn, st>>>(S, k, X, ctx->dev_status);
    PSC_LAUNCH_CHECK(ctx);
    return 0;
  }
  double* D = X;   // R11^{-T} of the current block step, in the first CB x CB of X (overwritten below)
  const int psmem = (CB + 64) * (CB + 1) * (int)sizeof(double);
  const int usmem = 2 * CB * (64 + 1) * (int)sizeof(double);
  PSC_CUDA(ctx, cudaFuncSetAttribute(k_potrf_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, psmem));
  PSC_CUDA(ctx, cudaFuncSetAttribute(k_potrf_update, cudaFuncAttributeMaxDynamicSharedMemorySize, usmem));
  for (int j0 = 0; j0 < k; j0 += CB) {
    const int nb = std::min(CB, k - j0);
    k_potrf_diag<<<1, 256, 0, st>>>(S, k, j0, D, ctx->dev_status);
    PSC_LAUNCH_CHECK(ctx);
    const int m = k - j0 - nb;
    if (m <= 0) break;
    k_potrf_panel<<<psc_div_up(m, 64), 256, psmem, st>>>(S, k, j0, D);
    PSC_LAUNCH_CHECK(ctx);
    const int t = psc_div_up(m, 64);
    k_potrf_update<<<dim3(t, t), 256, usmem, st>>>(S, k, j0);
    PSC_LAUNCH_CHECK(ctx);
  }
  k_tril_zero<<<std::max(1, std::min(592, psc_div_up((long)k * k, 256))), 256, 0, st>>>(S, k);
  PSC_LAUNCH_CHECK(ctx);
  // staged columns per chunk: 16, fewer when 8 b vectors + 16 columns of k
  // rows exceed 200 KB of shared memory
  const int ch = (int)std::max<long>(1, std::min<long>(16, ((200L * 1024 / 8) - 8L * k) / (k + 1)));
  const size_t tdyn = ((size_t)(8 + ch) * k + ch) * sizeof(double);
  PSC_REQUIRE(ctx, tdyn <= 227 * 1024, "chol_inv: k too large for the triangular inverse");
  if (tdyn > 48 * 1024)
    PSC_CUDA(ctx, cudaFuncSetAttribute(k_trtri_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tdyn));
  k_trtri_warp<<<psc_div_up(k, 8), 256, tdyn, st>>>(S, k, ch, X);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

// ---------------------------------------------------------------------------
// Symmetric eigensolver (ascending eigenvalues, orthonormal eigenvectors) of
// the symmetrised matrix (A + A^T) / 2:
//   1. k_sytrd: Householder reduction to tridiagonal form T = Q^T A Q in one
//      CTA, the matrix in shared memory up to k = 153 and in L2-resident
//      scratch beyond.  Step j reflects rows/columns j+1..k-1 with
//      H_j = I - tau_j v_j v_j^T, v_j[j+1] = 1, chosen so that H_j zeroes
//      A[j+2:, j] (dlarfg's Householder vector); the trailing block takes
//      the rank-2 update A <- A - v w^T - w v^T with p = tau A v and
//      w = p - (tau/2)(p.v) v.  Three barriers per step: partial products
//      A v over column groups, p and p.v, the rank-2 update; warp 0 builds
//      reflector j+1 inside the update, right after column j+1.
//   2. all eigenvalues of T by Sturm-count multisection and its eigenvectors
//      Z by inverse iteration (lanczos.cu), eigenvalues closer than 1e-3 |T|
//      orthogonalised against each other inside one warp;
//   3. k_ormtr: eigenvectors Q Z = H_0 H_1 ... H_{k-3} Z, one warp per column
//      applying the reflectors from the last to the first, staged in shared
//      memory in chunks.
// Against the one-CTA cyclic Jacobi solver this replaces (two barriers per
// rotation round, (k-1) rounds per sweep, 5-10 sweeps) the reduction takes
// 3 (k-2) barriers in all.
// ---------------------------------------------------------------------------
constexpr int SY_GMAX = 8;   // column groups of the partial products A v

static size_t sytrd_smem_doubles(int k, bool on_chip) {
  return (on_chip ? (size_t)k * k : 0) + (size_t)(3 + SY_GMAX) * k;
}

// Reflector j from column j below the diagonal (one warp): v -> v (shared)
// and hv column j (rows j+1..k-1), d_j, e_j = beta -> ab, tau_j -> tau and
// *s_t.  Off chip hv is A, so every lane reads x[i] before it writes hv[i].
__device__ __forceinline__ void sy_reflector(const double* A, int k, int j, double* __restrict__ hv, double* v,
                                             double* __restrict__ ab, double* __restrict__ tau, double* s_t,
                                             int lane) {
  const int L = k - j - 1;
  const double* x = A + (j + 1) + (long)j * k;
  const double alpha = x[0];   // read by every lane before lane 0 overwrites it (off chip)
  const double dj = A[j + (long)j * k];
  double sig = 0.0;
  for (int i = 1 + lane; i < L; i += 32) sig += x[i] * x[i];
  sig = psc_warp_sum(sig);
  double t = 0.0, beta = alpha, scal = 0.0;
  if (sig > 0.0) {
    beta = -copysign(sqrt(alpha * alpha + sig), alpha);
    t = (beta - alpha) / beta;
    scal = 1.0 / (alpha - beta);
  }
  double* hj = hv + (j + 1) + (long)j * k;
  for (int i = lane; i < L; i += 32) {
    const double vi = i == 0 ? 1.0 : x[i] * scal;
    v[i] = vi;
    hj[i] = vi;
  }
  if (lane == 0) {
    ab[2 * j] = dj;
    ab[2 * j + 1] = beta;
    tau[j] = t;
    *s_t = t;
  }
}

template <int NT>
__global__ void __launch_bounds__(NT)
k_sytrd(const double* __restrict__ Ain, int k, int on_chip, double* __restrict__ hv, double* __restrict__ ab,
        double* __restrict__ tau) {
  extern __shared__ double sm[];
  constexpr int NW = NT / 32;
  __shared__ double red[NW];
  // v and tau by the parity of j: warp 0 builds reflector j+1 while the other
  // warps still apply reflector j
  __shared__ double s_tau[2];
  double* A = on_chip ? sm : hv;   // off chip the reflectors overwrite the columns they annihilated
  double* vb = sm + (on_chip ? (size_t)k * k : 0);   // [2][k]
  double* p = vb + 2 * k;
  double* part = p + k;            // [SY_GMAX][k]
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int c = w; c < k; c += NW)
    for (int r = lane; r < k; r += 32) {
      const long e = r + (long)c * k;
      A[e] = (r == c) ? Ain[e] : 0.5 * (Ain[e] + Ain[c + (long)r * k]);
    }
  __syncthreads();
  if (k > 2 && w == 0) sy_reflector(A, k, 0, hv, vb, ab, tau, &s_tau[0], lane);
  __syncthreads();
  for (int j = 0; j + 2 < k; ++j) {
    const int L = k - j - 1;   // order of the trailing block
    double* A22 = A + (j + 1) + (long)(j + 1) * k;
    const double* v = vb + (j & 1) * k;
    double* vn = vb + ((j + 1) & 1) * k;
    const bool next = j + 3 < k;   // reflector j+1 exists
    const double t = s_tau[j & 1];
    if (t != 0.0) {   // the same branch in every thread
      // partial products sum_{c = g mod G} A22[i, c] v[c]
      const int R = min(NT, (L + 31) & ~31);
      const int G = min(SY_GMAX, NT / R);
      {
        const int r0 = tid % R, g = tid / R;
        if (g < G)
          for (int i = r0; i < L; i += R) {
            double s = 0.0;
            for (int c = g; c < L; c += G) s += A22[i + (long)c * k] * v[c];
            part[g * k + i] = s;
          }
      }
      __syncthreads();
      double q = 0.0;
      for (int i = tid; i < L; i += NT) {
        double s = 0.0;
        for (int g = 0; g < G; ++g) s += part[g * k + i];
        s *= t;
        p[i] = s;
        q += s * v[i];
      }
      q = psc_warp_sum(q);
      if (lane == 0) red[w] = q;
      __syncthreads();
      double pv = 0.0;
      for (int i = 0; i < NW; ++i) pv += red[i];
      const double K = 0.5 * t * pv;
      // rank-2 update; warp 0 takes column 0 (column j+1 of A) first and
      // builds reflector j+1 from it before its other columns
      for (int c = w; c < L; c += NW) {
        const double vc = v[c], wc = p[c] - K * vc;
        double* col = A22 + (long)c * k;
        for (int r = lane; r < L; r += 32) {
          const double vr = v[r];
          col[r] -= vr * wc + (p[r] - K * vr) * vc;
        }
        if (c == 0 && next) {
          __syncwarp();
          sy_reflector(A, k, j + 1, hv, vn, ab, tau, &s_tau[(j + 1) & 1], lane);
        }
      }
    } else if (w == 0 && next) {   // H_j = I: column j+1 is unchanged
      sy_reflector(A, k, j + 1, hv, vn, ab, tau, &s_tau[(j + 1) & 1], lane);
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (k >= 2) {
      ab[2 * (k - 2)] = A[(k - 2) + (long)(k - 2) * k];
      ab[2 * (k - 2) + 1] = A[(k - 1) + (long)(k - 2) * k];
    }
    ab[2 * (k - 1)] = A[(k - 1) + (long)(k - 1) * k];
    ab[2 * (k - 1) + 1] = 0.0;
  }
}

// The same reduction for matrices too large for one CTA's shared memory
// (153 < k <= ~420): a cluster of SY_CL CTAs holds the symmetrised matrix in
// their shared memory, column c in CTA c mod SY_CL (cyclic, so the trailing
// block stays spread over all of them).  Step j:
//   the owner of column j builds reflector j (one warp, as sy_reflector) and
//   writes it to hv / ab / tau;                               cluster barrier
//   every CTA copies v and tau from the owner's shared memory, and forms the
//   partial products of its columns, part = sum_c A[:, c] v_c; cluster barrier
//   every CTA sums the SY_CL partials in rank order (distributed shared
//   memory, the same order everywhere), p = tau part, K = tau (p.v) / 2, and
//   applies the rank-2 update A -= v w^T + w v^T (w = p - K v) to its columns.
// Two cluster barriers per step instead of three block barriers over L2.
constexpr int SY_CL = 8;
constexpr int SY_CNT = 512;

static size_t sytrd_cl_smem_doubles(int k) {
  return (size_t)((k + SY_CL - 1) / SY_CL) * k + 3 * (size_t)k;
}

__global__ void __cluster_dims__(SY_CL, 1, 1) __launch_bounds__(SY_CNT)
k_sytrd_cl(const double* __restrict__ Ain, int k, double* __restrict__ hv, double* __restrict__ ab,
           double* __restrict__ tau) {
  extern __shared__ double sm[];
  __shared__ double red[SY_CNT / 32];
  __shared__ double s_t;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int ncl = (k + SY_CL - 1) / SY_CL;
  double* A = sm;                        // [ncl][k]: local column lc is global column rank + SY_CL lc
  double* vb = A + (size_t)ncl * k;      // reflector, entry i = row j+1+i
  double* part = vb + k;                 // this CTA's partial products (row j+1+i at i)
  double* pf = part + k;                 // p
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int lc = w; lc < ncl; lc += SY_CNT / 32) {
    const int c = rank + SY_CL * lc;
    if (c >= k) continue;
    for (int r = lane; r < k; r += 32)
      A[(long)lc * k + r] = (r == c) ? Ain[r + (long)c * k] : 0.5 * (Ain[r + (long)c * k] + Ain[c + (long)r * k]);
  }
  __syncthreads();
  for (int j = 0; j + 2 < k; ++j) {
    const int L = k - j - 1;
    const int owner = j % SY_CL;
    if (rank == owner && w == 0) {
      // reflector j from column j below the diagonal
      const double* x = A + (long)(j / SY_CL) * k + (j + 1);
      const double alpha = x[0];
      double sig = 0.0;
      for (int i = 1 + lane; i < L; i += 32) sig += x[i] * x[i];
      sig = psc_warp_sum(sig);
      double t = 0.0, beta = alpha, scal = 0.0;
      if (sig > 0.0) {
        beta = -copysign(sqrt(alpha * alpha + sig), alpha);
        t = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      for (int i = lane; i < L; i += 32) {
        const double vi = i == 0 ? 1.0 : x[i] * scal;
        vb[i] = vi;
        hv[(j + 1 + i) + (long)j * k] = vi;
      }
      if (lane == 0) {
        ab[2 * j] = A[(long)(j / SY_CL) * k + j];
        ab[2 * j + 1] = beta;
        tau[j] = t;
        s_t = t;
      }
    }
    cl.sync();
    const double t = *cl.map_shared_rank(&s_t, owner);
    if (rank != owner) {
      const double* rv = cl.map_shared_rank(vb, owner);
      for (int i = tid; i < L; i += SY_CNT) vb[i] = rv[i];
    }
    __syncthreads();
    const int lc0 = (j + 1 - rank + SY_CL - 1) / SY_CL;   // first local column with c >= j+1
    if (t != 0.0) {
      for (int i = tid; i < L; i += SY_CNT) {
        double acc = 0.0;
        for (int lc = lc0; lc < ncl; ++lc) {
          const int c = rank + SY_CL * lc;
          if (c >= k) break;
          acc += A[(long)lc * k + (j + 1 + i)] * vb[c - (j + 1)];
        }
        part[i] = acc;
      }
    }
    cl.sync();
    if (t != 0.0) {
      double q = 0.0;
      for (int i = tid; i < L; i += SY_CNT) {
        double acc = 0.0;
        for (int r = 0; r < SY_CL; ++r) acc += cl.map_shared_rank(part, r)[i];
        const double pi = t * acc;
        pf[i] = pi;
        q += pi * vb[i];
      }
      q = psc_warp_sum(q);
      if (lane == 0) red[w] = q;
      __syncthreads();
      double pv = 0.0;
      for (int i = 0; i < SY_CNT / 32; ++i) pv += red[i];
      const double K = 0.5 * t * pv;
      for (int lc = lc0 + w; lc < ncl; lc += SY_CNT / 32) {
        const int c = rank + SY_CL * lc;
        if (c >= k) continue;
        const int ci = c - (j + 1);
        const double vc = vb[ci], wc = pf[ci] - K * vc;
        double* col = A + (long)lc * k + (j + 1);
        for (int r = lane; r < L; r += 32) {
          const double vr = vb[r];
          col[r] -= vr * wc + (pf[r] - K * vr) * vc;
        }
      }
    }
    __syncthreads();
  }
  // the last 2 x 2 block
  if (tid == 0 && k >= 2) {
    if (rank == (k - 2) % SY_CL) {
      ab[2 * (k - 2)] = A[(long)((k - 2) / SY_CL) * k + (k - 2)];
      ab[2 * (k - 2) + 1] = A[(long)((k - 2) / SY_CL) * k + (k - 1)];
    }
    if (rank == (k - 1) % SY_CL) {
      ab[2 * (k - 1)] = A[(long)((k - 1) / SY_CL) * k + (k - 1)];
      ab[2 * (k - 1) + 1] = 0.0;
    }
  }
  cl.sync();   // no CTA leaves while others may still read its shared memory
}

// out = H_0 H_1 ... H_{k-3} Z (Z k x k, ld k).  A CTA owns OR_NW columns, one
// warp each; the whole CTA stages the reflectors OR_CH at a time in shared
// memory (one round of independent L2 loads per chunk instead of two
// dependent ones per reflector), then every warp applies them to its column.
constexpr int OR_NW = 8, OR_CH = 16;

static size_t ormtr_smem_bytes(int k) { return (size_t)(OR_NW + OR_CH) * k * sizeof(double); }

__global__ void __launch_bounds__(OR_NW * 32)
k_ormtr(const double* __restrict__ hv, const double* __restrict__ tau, int k, const double* __restrict__ Z,
        double* __restrict__ out) {
  extern __shared__ double sm[];
  __shared__ double ts[OR_CH];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int col = blockIdx.x * OR_NW + w;
  double* z = sm + (size_t)w * k;
  double* vs = sm + (size_t)OR_NW * k;   // [OR_CH][k]
  if (col < k)
    for (int i = lane; i < k; i += 32) z[i] = Z[i + (long)col * k];
  for (int j1 = k - 3; j1 >= 0; j1 -= OR_CH) {
    const int j0 = max(0, j1 - OR_CH + 1);
    __syncthreads();   // the previous chunk is consumed
    for (int c = w; c <= j1 - j0; c += OR_NW) {
      const int j = j0 + c;
      for (int i = j + 1 + lane; i < k; i += 32) vs[(size_t)c * k + i] = hv[i + (long)j * k];
      if (lane == 0) ts[c] = tau[j];
    }
    __syncthreads();
    if (col < k)
      for (int j = j1; j >= j0; --j) {
        const double t = ts[j - j0];
        if (t == 0.0) continue;
        const double* vj = vs + (size_t)(j - j0) * k;   // rows j+1..k-1
        double s = 0.0;
        for (int i = j + 1 + lane; i < k; i += 32) s += vj[i] * z[i];
        s = psc_warp_sum(s) * t;
        for (int i = j + 1 + lane; i < k; i += 32) z[i] -= s * vj[i];
        __syncwarp();
      }
  }
  if (col < k)
    for (int i = lane; i < k; i += 32) out[i + (long)col * k] = z[i];
}

int psc_syev_impl(psc_ctx* ctx, double* A, int k, double* evals, double* evecs, cudaStream_t st) {
  PSC_REQUIRE(ctx, k >= 1 && k <= PSC_MAX_K, "syev: k out of range");
  if (psc_ensure_dense(ctx, k)) return 1;
  const size_t kk = (size_t)k * k;
  double* hv = ctx->eig_work;   // reflectors (and the matrix itself when it is not on chip)
  double* Z = hv + kk;       // eigenvectors of T
  double* ab = Z + kk;       // T: diagonal ab[2i], off-diagonal ab[2i+1]
  double* tau = ab + 2 * k;
  const bool on_chip = sytrd_smem_doubles(k, true) * sizeof(double) <= 200 * 1024;
  const size_t dyn_cl = sytrd_cl_smem_doubles(k) * sizeof(double);
  const bool clustered = !on_chip && k >= 3 && dyn_cl <= 200 * 1024;
  const size_t dyn = sytrd_smem_doubles(k, on_chip) * sizeof(double);
#define PSC_SYTRD(NTH)                                                                                      \
  {                                                                                                         \
    if (dyn > 48 * 1024)                                                                                    \
      PSC_CUDA(ctx, cudaFuncSetAttribute(k_sytrd<NTH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn)); \
    k_sytrd<NTH><<<1, NTH, dyn, st>>>(A, k, on_chip ? 1 : 0, hv, ab, tau);                                  \
  }
  if (clustered) {
    PSC_CUDA(ctx, cudaFuncSetAttribute(k_sytrd_cl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_cl));
    k_sytrd_cl<<<SY_CL, SY_CNT, dyn_cl, st>>>(A, k, hv, ab, tau);
  } else if (!on_chip) PSC_SYTRD(1024)
  else if (k <= 96) PSC_SYTRD(256)
  else PSC_SYTRD(512)
#undef PSC_SYTRD
  PSC_LAUNCH_CHECK(ctx);
  int rc = psc_tridiag_eig_impl(ctx, ab, k, k, evals, Z, k, 1e-3, st);
  if (rc) return rc;
  const size_t dyn2 = ormtr_smem_bytes(k);
  if (dyn2 > 48 * 1024)
    PSC_CUDA(ctx, cudaFuncSetAttribute(k_ormtr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn2));
  k_ormtr<<<psc_div_up(k, OR_NW), OR_NW * 32, dyn2, st>>>(hv, tau, k, Z, evecs);
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
    rc = psc_chol_inv_dev(ctx, ctx->gram, k, ctx->tri, st);
    if (rc) return rc;
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
