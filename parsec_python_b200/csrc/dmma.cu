// FP64 tensor-core (DMMA, mma.sync m8n8k4 .f64) kernels for the tall
// products of the Rayleigh-Ritz step, for FP64 blocks and for FP32 blocks
// that need products without the FP32 accumulation of tcgen05 (every FP32
// input is exact in FP64, the products and sums are FP64, the result is
// rounded once).  Blackwell's tcgen05 has no FP64 kind; DMMA is the FP64
// tensor path.
//
//   k_gram_dmma   S = W^T W and K = W^T V: one CTA per (upper-triangle pair
//                 of 64-column tiles, chunk of rows); warps 0-3 accumulate
//                 the S tile, warps 4-7 the K tile, each a 32 x 32 block of
//                 4 x 4 DMMA tiles; 32 rows per stage through shared memory,
//                 the next stage's loads in flight in registers.  Per-chunk
//                 FP64 partial tiles, summed over the chunks in a fixed
//                 order by k_gram_dmma_final.
//   k_gemm_dmma   Out (n x kout) = W (n x k) T (k x kout): 128 rows x 64
//                 columns per CTA, 8 warps of 32 x 32, T staged 32 rows at a
//                 time.
//
// Fragment layout of mma.m8n8k4.row.col.f64 (lane l): A[l / 4][l % 4],
// B[l % 4][l / 4], C and D [l / 4][2 (l % 4) + {0, 1}].
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>
#include <vector>

namespace {

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

constexpr int GT = 64;       // Gram output tile
constexpr int GS = 32;       // rows per stage
constexpr int GP = GS + 4;   // padded row count of a staged column: the fragment loads
                             // (8 columns x 4 rows per instruction) take two wavefronts
constexpr int GNT = 256;
constexpr int GPER = GT * GS / GNT;   // staged values per thread and tile

template <typename T>
struct GramLoad {
  T v[3][GPER];
};

// tile m (0: W columns of tile i, 1: W columns of tile j, 2: V columns of
// tile j) of rows r0 .. r0 + GS - 1: element e = tid + GNT u is row e % GS
// of column e / GS (consecutive threads read consecutive rows)
template <typename T>
__device__ __forceinline__ void gram_load(const T* __restrict__ W, const T* __restrict__ V, long ld, int k, long r0,
                                          long r1, int ci, int cj, bool diag, GramLoad<T>& g) {
#pragma unroll
  for (int u = 0; u < GPER; ++u) {
    const int e = threadIdx.x + GNT * u;
    const int r = e % GS, c = e / GS;
    const long row = r0 + r;
    const bool ok = row < r1;
    g.v[0][u] = (ok && ci + c < k) ? W[row + (long)(ci + c) * ld] : T(0);
    g.v[1][u] = (ok && !diag && cj + c < k) ? W[row + (long)(cj + c) * ld] : T(0);
    g.v[2][u] = (ok && cj + c < k) ? V[row + (long)(cj + c) * ld] : T(0);
  }
}

}  // namespace

template <typename T>
__global__ void __launch_bounds__(GNT)
k_gram_dmma(const T* __restrict__ W, const T* __restrict__ V, long ld, int k, long n, long chunk,
            const int2* __restrict__ pairs, double* __restrict__ partS, double* __restrict__ partK) {
  extern __shared__ double gsm[];
  double (*sI)[GP] = reinterpret_cast<double (*)[GP]>(gsm);              // [GT][GP] W, tile i
  double (*sJ)[GP] = reinterpret_cast<double (*)[GP]>(gsm + GT * GP);    // W, tile j
  double (*sV)[GP] = reinterpret_cast<double (*)[GP]>(gsm + 2 * GT * GP);  // V, tile j
  const int2 pr = pairs[blockIdx.x];
  const int ci = pr.x * GT, cj = pr.y * GT;
  const bool diag = pr.x == pr.y;
  const long r0 = (long)blockIdx.y * chunk;
  const long r1 = min(n, r0 + chunk);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int which = warp >> 2;                     // 0: S, 1: K
  const int wr = (warp >> 1) & 1, wc = warp & 1;   // 32 x 32 block of the warp
  double (*Bt)[GP] = which ? sV : (diag ? sI : sJ);
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  GramLoad<T> g;
  if (r0 < r1) gram_load(W, V, ld, k, r0, r1, ci, cj, diag, g);
  for (long rb = r0; rb < r1; rb += GS) {
    __syncthreads();   // the previous stage's fragments are read
#pragma unroll
    for (int u = 0; u < GPER; ++u) {
      const int e = threadIdx.x + GNT * u;
      const int r = e % GS, c = e / GS;
      sI[c][r] = (double)g.v[0][u];
      if (!diag) sJ[c][r] = (double)g.v[1][u];
      sV[c][r] = (double)g.v[2][u];
    }
    __syncthreads();
    if (rb + GS < r1) gram_load(W, V, ld, k, rb + GS, r1, ci, cj, diag, g);
#pragma unroll
    for (int ks = 0; ks < GS / 4; ++ks) {
      const int rr = 4 * ks + (lane & 3);
      double a[4], b[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        a[m] = sI[wr * 32 + m * 8 + (lane >> 2)][rr];
        b[m] = Bt[wc * 32 + m * 8 + (lane >> 2)][rr];
      }
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int q = 0; q < 4; ++q) dmma(acc[m][q][0], acc[m][q][1], a[m], b[q]);
    }
  }
  double* out = (which ? partK : partS) + (long)blockIdx.y * k * k;
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gi = ci + wr * 32 + m * 8 + (lane >> 2);
        const int gj = cj + wc * 32 + q * 8 + 2 * (lane & 3) + h;
        if (gi < k && gj < k) out[gi + (long)gj * k] = acc[m][q][h];
      }
}

// S, K = sums over the chunks (one warp per entry, lanes take every 32nd
// chunk, then a fixed shuffle tree).  Only tile pairs (i <= j) were formed:
// an entry below the diagonal tiles takes its mirror, entries of diagonal
// tiles are symmetrised as 0.5 (X + X^T).
__global__ void k_gram_dmma_final(const double* __restrict__ partS, const double* __restrict__ partK, int nchunk,
                                  int k, double* __restrict__ S, double* __restrict__ K) {
  const long kk = (long)k * k;
  const int lane = threadIdx.x & 31;
  const long nwarps = (long)gridDim.x * (blockDim.x >> 5);
  for (long e = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < 2 * kk; e += nwarps) {
    const bool isK = e >= kk;
    const long f = isK ? e - kk : e;
    const int i = (int)(f % k), j = (int)(f / k);
    const int ti = i / GT, tj = j / GT;
    const long src = ti <= tj ? f : j + (long)i * k;   // an entry of an upper tile pair
    const long mir = j + (long)i * k;
    const double* P = isK ? partK : partS;
    double s = 0.0, u = 0.0;
    for (int c = lane; c < nchunk; c += 32) {
      s += P[(long)c * kk + src];
      if (ti == tj) u += P[(long)c * kk + mir];
    }
    s = psc_warp_sum(s);
    if (ti == tj) u = psc_warp_sum(u);
    if (lane == 0) (isK ? K : S)[f] = ti == tj ? 0.5 * (s + u) : s;
  }
}

namespace {
constexpr int MR = 128;       // rows of Out per CTA
constexpr int MC = 64;        // columns of Out per CTA
constexpr int MK = 32;        // reduction entries per stage
constexpr int MWP = MR + 8;   // padded row count of a staged W column (two wavefronts per fragment load)
constexpr int MTP = MK + 4;   // padded reduction count of a staged T column
constexpr int MPER = MR * MK / GNT;   // W values staged per thread and stage
}  // namespace

template <typename T>
__global__ void __launch_bounds__(GNT)
k_gemm_dmma(const T* __restrict__ W, long ldw, int k, const double* __restrict__ Tm, int kout, T* __restrict__ O,
            long ldo, long n) {
  extern __shared__ double msm[];
  double (*sW)[MWP] = reinterpret_cast<double (*)[MWP]>(msm);              // [MK][MWP]: reduction index, row
  double (*sT)[MTP] = reinterpret_cast<double (*)[MTP]>(msm + MK * MWP);   // [MC][MTP]: column, reduction index
  const long row0 = (long)blockIdx.y * MR;
  const int col0 = blockIdx.x * MC;   // column blocks of one row block run side by side and share W through L2
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wr = warp >> 1, wc = warp & 1;   // rows 32 wr .., columns 32 wc ..
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  T wv[MPER];
  auto load_w = [&](int i0) {
#pragma unroll
    for (int u = 0; u < MPER; ++u) {
      const int e = threadIdx.x + GNT * u;
      const int r = e % MR, i = e / MR;
      const long row = row0 + r;
      wv[u] = (row < n && i0 + i < k) ? W[row + (long)(i0 + i) * ldw] : T(0);
    }
  };
  load_w(0);
  for (int i0 = 0; i0 < k; i0 += MK) {
    __syncthreads();
#pragma unroll
    for (int u = 0; u < MPER; ++u) {
      const int e = threadIdx.x + GNT * u;
      sW[e / MR][e % MR] = (double)wv[u];
    }
    for (int e = threadIdx.x; e < MK * MC; e += GNT) {
      const int i = e % MK, c = e / MK;
      sT[c][i] = (i0 + i < k && col0 + c < kout) ? Tm[(i0 + i) + (long)(col0 + c) * k] : 0.0;
    }
    __syncthreads();
    if (i0 + MK < k) load_w(i0 + MK);
#pragma unroll
    for (int ks = 0; ks < MK / 4; ++ks) {
      const int ii = 4 * ks + (lane & 3);
      double a[4], b[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        a[m] = sW[ii][wr * 32 + m * 8 + (lane >> 2)];
        b[m] = sT[wc * 32 + m * 8 + (lane >> 2)][ii];
      }
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int q = 0; q < 4; ++q) dmma(acc[m][q][0], acc[m][q][1], a[m], b[q]);
    }
  }
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long row = row0 + wr * 32 + m * 8 + (lane >> 2);
        const int c = col0 + wc * 32 + q * 8 + 2 * (lane & 3) + h;
        if (row < n && c < kout) O[row + (long)c * ldo] = (T)acc[m][q][h];
      }
}

int psc_gram_pair_dmma(psc_ctx* ctx, int dtype, const void* W, const void* V, long ld, int k, double* S, double* K,
                       cudaStream_t st) {
  const long n = ctx->n;
  const int tiles = (k + GT - 1) / GT;
  const int npair = tiles * (tiles + 1) / 2;
  if (ctx->dm_pairs_k != k) {
    std::vector<int2> hp;
    for (int a = 0; a < tiles; ++a)
      for (int b = a; b < tiles; ++b) hp.push_back(make_int2(a, b));
    if ((int)hp.size() > ctx->dm_pairs_cap) {
      psc_dfree(ctx->dm_pairs);
      ctx->dm_pairs = nullptr;
      ctx->dm_pairs_cap = 0;
      PSC_CUDA(ctx, psc_dmalloc(&ctx->dm_pairs, hp.size() * sizeof(int2)));
      ctx->dm_pairs_cap = (int)hp.size();
    }
    PSC_CUDA(ctx, cudaMemcpy(ctx->dm_pairs, hp.data(), hp.size() * sizeof(int2), cudaMemcpyHostToDevice));
    ctx->dm_pairs_k = k;
  }
  // about four waves of two CTAs per SM, within the partial buffer
  int nchunk = std::max(1, std::min(ctx->gram_blocks / 2, (148 * 8 + npair - 1) / npair));
  nchunk = (int)std::min<long>(nchunk, std::max<long>(1, n / GS));
  const long chunk = ((n + nchunk - 1) / nchunk + GS - 1) / GS * GS;
  nchunk = (int)((n + chunk - 1) / chunk);
  double* partS = ctx->gram_partial;
  double* partK = ctx->gram_partial + (size_t)nchunk * k * k;
  const size_t smem = 3 * (size_t)GT * GP * sizeof(double);
  dim3 grid(npair, nchunk);
  if (dtype == PSC_F64) {
    PSC_CUDA(ctx, cudaFuncSetAttribute(k_gram_dmma<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_gram_dmma<double><<<grid, GNT, smem, st>>>((const double*)W, (const double*)V, ld, k, n, chunk,
                                                  (const int2*)ctx->dm_pairs, partS, partK);
  } else {
    PSC_CUDA(ctx, cudaFuncSetAttribute(k_gram_dmma<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_gram_dmma<float><<<grid, GNT, smem, st>>>((const float*)W, (const float*)V, ld, k, n, chunk,
                                                 (const int2*)ctx->dm_pairs, partS, partK);
  }
  PSC_LAUNCH_CHECK(ctx);
  const long kk = (long)k * k;
  k_gram_dmma_final<<<std::max(1, (int)std::min<long>(148 * 8, (2 * kk + 7) / 8)), 256, 0, st>>>(partS, partK,
                                                                                               nchunk, k, S, K);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

int psc_gemm_tall_dmma(psc_ctx* ctx, int dtype, const void* W, long ldw, int k, const double* Tm, int kout, void* O,
                       long ldo, cudaStream_t st) {
  const size_t smem = ((size_t)MK * MWP + (size_t)MC * MTP) * sizeof(double);
  dim3 grid(psc_div_up(kout, MC), psc_div_up(ctx->n, MR));
  PSC_REQUIRE(ctx, grid.y <= 65535u, "gemm: too many row blocks");
  if (dtype == PSC_F64) {
    PSC_CUDA(ctx, cudaFuncSetAttribute(k_gemm_dmma<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_gemm_dmma<double><<<grid, GNT, smem, st>>>((const double*)W, ldw, k, Tm, kout, (double*)O, ldo, ctx->n);
  } else {
    PSC_CUDA(ctx, cudaFuncSetAttribute(k_gemm_dmma<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_gemm_dmma<float><<<grid, GNT, smem, st>>>((const float*)W, ldw, k, Tm, kout, (float*)O, ldo, ctx->n);
  }
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}
