// Tensor-core Gram pair for the mixed-precision subspace step:
// S = W^T W and K = W^T V (V = H W) from FP32 blocks, on tcgen05 with TF32
// operands and FP32 accumulation in tensor memory, with the three-term
// split-precision correction x = hi + lo (hi = tf32(x), lo = tf32(x - hi)):
//   W^T V ~ hi(W)^T hi(V) + hi(W)^T lo(V) + lo(W)^T hi(V),
// which keeps FP32-level accuracy (the dropped lo*lo term is ~2^-22).
// Replaces the dense products of Rayleighritz.py:4-30 / chefsi1.py:43-67 in
// the mixed-precision path; the FP64 path keeps the CUDA-core kernels.
//
// Grid: (pair of 128-column tiles, upper triangle) x (chunk of the n rows).
// Each CTA streams its rows through a two-deep shared-memory ring, 32 rows
// (one 128-byte swizzle row of FP32) per stage, the next stage's loads in
// flight in registers while the current one is stored; its threads load and split
// the tiles into hi/lo copies in the canonical K-major 128-byte-swizzled
// layout, one elected thread issues the MMAs and commits them to an
// mbarrier.  The W_b and V_b tiles of a stage sit next to each other in
// shared memory, so one MMA of N = 2 x tile width (K = 8) yields the S and
// K blocks side by side in tensor memory: three MMAs per K step (hi hi,
// hi lo, lo hi), each reading its A tile once for both products.  Partial FP32
// tiles go to global memory and are summed over the chunks in FP64.
// The tensor cores' FP32 accumulation rounds toward zero, so a long chunk
// biases every entry towards zero (about 1e-4 relative at 7,000 rows).  The
// diagonal entries (column norms and Rayleigh quotients, which set the
// density's normalisation and the eigenvalue sum) are therefore recomputed
// exactly: the CTAs of diagonal tile pairs sum w_j^2 and w_j v_j in FP64
// from the same FP32 registers they split, and the final kernel uses those.
// Every wait is bounded by the context's wait limit; on a timeout the kernel
// drains the MMAs it issued and records status word 5.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>

namespace {
constexpr int TC_NT = 256;              // 8 warps: loads in flight; warps 0-3 also drain TMEM
constexpr int TROWS = 128;               // tile rows (matrix columns), = MMA M
constexpr int KSTAGE = 32;               // reduction rows per stage (128 bytes of FP32)
constexpr int TILE_BYTES = TROWS * 128;  // 16 KB
constexpr int NTILES = 6;                // [W_b V_b] hi, [W_b V_b] lo, A hi, A lo
constexpr int BUF_BYTES = NTILES * TILE_BYTES;
constexpr int TMEM_COLS = 256;           // S accumulator at column 0, K at column N

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (start >> 4, LBO 1 (unused by swizzled K-major), SBO
// 1024 >> 4, descriptor version 1, layout type 2 = SWIZZLE_128B)
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)(1024u >> 4) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;
  return d;
}

// instruction descriptor, kind::tf32: D F32, A and B TF32, both K-major, N, M = 128
__host__ __device__ constexpr uint32_t idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TROWS >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, long limit) {
  for (long i = 0; i < limit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// One tile of a stage: rows [0, nrows) x 32 reduction entries (rows = matrix
// columns col0 + r, valid below `valid`; reduction entries n0 .. n0+31 below
// n_end).  Each thread owns up to PER 16-byte pieces; all loads of a stage
// are issued before any is used, then split into hi/lo and stored swizzled.
constexpr int PER = TROWS * 8 / TC_NT;   // pieces per thread and tile

struct TileLoad {
  float4 v[PER];
};

__device__ __forceinline__ void tile_load(const float* __restrict__ M, long ld, int col0, int valid, int nrows,
                                          long n0, long n_end, bool vec, TileLoad& t) {
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int i = threadIdx.x + u * TC_NT;
    const int row = i >> 3, c = i & 7;
    const long nn = n0 + 4 * c;
    float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
    if (row < nrows && row < valid && nn < n_end) {
      const float* src = M + (long)(col0 + row) * ld + nn;
      if (vec && nn + 3 < n_end) {
        x = __ldg(reinterpret_cast<const float4*>(src));
      } else {
        x.x = __ldg(src);
        if (nn + 1 < n_end) x.y = __ldg(src + 1);
        if (nn + 2 < n_end) x.z = __ldg(src + 2);
        if (nn + 3 < n_end) x.w = __ldg(src + 3);
      }
    }
    t.v[u] = x;
  }
}

__device__ __forceinline__ void tile_store_split(const TileLoad& t, int nrows, unsigned char* hi, unsigned char* lo) {
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int i = threadIdx.x + u * TC_NT;
    const int row = i >> 3, c = i & 7;
    if (row >= nrows) continue;
    const float4 x = t.v[u];
    float4 h, l;
    h.x = tf32_rna(x.x); l.x = tf32_rna(x.x - h.x);
    h.y = tf32_rna(x.y); l.y = tf32_rna(x.y - h.y);
    h.z = tf32_rna(x.z); l.z = tf32_rna(x.z - h.z);
    h.w = tf32_rna(x.w); l.w = tf32_rna(x.w - h.w);
    const int off = row * 128 + ((c ^ (row & 7)) << 4);
    *reinterpret_cast<float4*>(hi + off) = h;
    *reinterpret_cast<float4*>(lo + off) = l;
  }
}
}  // namespace

__global__ void __launch_bounds__(TC_NT, 1)
k_gram_tc(const float* __restrict__ W, const float* __restrict__ V, long ld, int k, long n, long chunk,
          const int2* __restrict__ pairs, float* __restrict__ part, double* __restrict__ dpart, long wait_limit,
          int* status) {
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5;
  // blockIdx.x = tile pair, blockIdx.y = row chunk: the pairs of one chunk
  // run side by side and stream the same rows, which they share through L2
  const int2 pr = pairs[blockIdx.x];
  const int mt = pr.x, nt = pr.y;
  const int col_a = mt * TROWS, col_b = nt * TROWS;
  const int valid_a = min(TROWS, k - col_a), valid_b = min(TROWS, k - col_b);
  const int N = (valid_b + 15) & ~15;   // MMA N: multiple of 16 for M = 128
  const bool same = mt == nt;
  const long n_begin = (long)blockIdx.y * chunk;
  const long n_end = min(n, n_begin + chunk);
  const int nstage = (int)((max(0L, n_end - n_begin) + KSTAGE - 1) / KSTAGE);
  const bool vec = ((ld & 3) == 0) && ((reinterpret_cast<uintptr_t>(W) & 15) == 0) &&
                   ((reinterpret_cast<uintptr_t>(V) & 15) == 0);

  if (threadIdx.x == 0) {
    s_fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const uint32_t tmem_s = tmem, tmem_k = tmem + N;
  const uint32_t idesc2 = idesc_tf32(2 * N);   // B = [W_b | V_b], D = [S | K]
  // exact FP64 diagonal sums of a diagonal tile pair: this thread's columns
  // are col_a + (threadIdx.x >> 3) + 32 u, u < PER
  double dsum_s[PER], dsum_k[PER];
#pragma unroll
  for (int u = 0; u < PER; ++u) dsum_s[u] = dsum_k[u] = 0.0;

  int last_commit = -1;   // thread 0: stage of the last MMA commit
  // the tiles of stage s+1 are loaded into registers while stage s is split,
  // stored and multiplied, so the HBM latency overlaps the tensor-core work
  TileLoad ta, tb, tk;
  if (nstage > 0) {
    tile_load(W, ld, col_a, valid_a, TROWS, n_begin, n_end, vec, ta);
    if (!same) tile_load(W, ld, col_b, valid_b, N, n_begin, n_end, vec, tb);
    tile_load(V, ld, col_b, valid_b, N, n_begin, n_end, vec, tk);
  }
  for (int s = 0; s < nstage; ++s) {
    const int b = s & 1;
    unsigned char* buf = sm + b * BUF_BYTES;
    // N rows of W_b followed by N rows of V_b (N is a multiple of 16, so the
    // V_b rows start on an 8-row swizzle group); a diagonal pair's A tile is
    // its W_b rows (the MMA's rows beyond N read V_b and land in discarded
    // accumulator rows)
    unsigned char* bs_hi = buf;
    unsigned char* bk_hi = buf + N * 128;
    unsigned char* bs_lo = buf + 2 * TILE_BYTES;
    unsigned char* bk_lo = bs_lo + N * 128;
    unsigned char* a_hi = same ? bs_hi : buf + 4 * TILE_BYTES;
    unsigned char* a_lo = same ? bs_lo : buf + 5 * TILE_BYTES;
    if (s >= 2 && threadIdx.x == 0) {
      // the MMAs of stage s-2 read this buffer: wait for their commit
      if (!mbar_wait(smem_u32(&mbar[b]), (uint32_t)(((s - 2) >> 1) & 1), wait_limit)) s_fail = 1;
    }
    __syncthreads();
    if (s_fail) break;
    {
      if (same) {
#pragma unroll
        for (int u = 0; u < PER; ++u) {
          const float4 a = ta.v[u], v = tk.v[u];
          dsum_s[u] = fma((double)a.x, (double)a.x, dsum_s[u]);
          dsum_s[u] = fma((double)a.y, (double)a.y, dsum_s[u]);
          dsum_s[u] = fma((double)a.z, (double)a.z, dsum_s[u]);
          dsum_s[u] = fma((double)a.w, (double)a.w, dsum_s[u]);
          dsum_k[u] = fma((double)a.x, (double)v.x, dsum_k[u]);
          dsum_k[u] = fma((double)a.y, (double)v.y, dsum_k[u]);
          dsum_k[u] = fma((double)a.z, (double)v.z, dsum_k[u]);
          dsum_k[u] = fma((double)a.w, (double)v.w, dsum_k[u]);
        }
      }
      if (same) {
        tile_store_split(ta, N, bs_hi, bs_lo);
      } else {
        tile_store_split(ta, TROWS, a_hi, a_lo);
        tile_store_split(tb, N, bs_hi, bs_lo);
      }
      tile_store_split(tk, N, bk_hi, bk_lo);
      if (s + 1 < nstage) {
        const long n1 = n_begin + (long)(s + 1) * KSTAGE;
        tile_load(W, ld, col_a, valid_a, TROWS, n1, n_end, vec, ta);
        if (!same) tile_load(W, ld, col_b, valid_b, N, n1, n_end, vec, tb);
        tile_load(V, ld, col_b, valid_b, N, n1, n_end, vec, tk);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
      const uint32_t bh = smem_u32(bs_hi), bl = smem_u32(bs_lo);
#pragma unroll
      for (int kk = 0; kk < KSTAGE / 8; ++kk) {
        const uint32_t o = kk * 32;   // 8 TF32 = 32 bytes along K inside the swizzled row
        const uint32_t acc = (s > 0 || kk > 0) ? 1u : 0u;
        mma_tf32(tmem_s, sw128_desc(ah + o), sw128_desc(bh + o), idesc2, acc);
        mma_tf32(tmem_s, sw128_desc(ah + o), sw128_desc(bl + o), idesc2, 1u);
        mma_tf32(tmem_s, sw128_desc(al + o), sw128_desc(bh + o), idesc2, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mbar[b]))
                   : "memory");
      last_commit = s;
    }
  }
  // the last commit covers every MMA issued before it; after a failed wait
  // the MMAs still in flight are drained before tensor memory is released
  if (threadIdx.x == 0 && last_commit >= 0) {
    const uint32_t bar = smem_u32(&mbar[last_commit & 1]), par = (uint32_t)((last_commit >> 1) & 1);
    if (s_fail || !mbar_wait(bar, par, wait_limit)) {
      s_fail = 1;
      mbar_wait(bar, par, PSC_DRAIN_WAIT);
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (same && !s_fail && nstage > 0) {
    // the 8 lanes that share a column (equal lane >> 3) sum their parts
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      for (int o = 1; o < 8; o <<= 1) {
        dsum_s[u] += __shfl_xor_sync(0xffffffffu, dsum_s[u], o);
        dsum_k[u] += __shfl_xor_sync(0xffffffffu, dsum_k[u], o);
      }
      const int row = (threadIdx.x >> 3) + u * (TC_NT / 8);
      if ((threadIdx.x & 7) == 0 && row < valid_a) {
        dpart[((long)blockIdx.y * 2 + 0) * k + col_a + row] = dsum_s[u];
        dpart[((long)blockIdx.y * 2 + 1) * k + col_a + row] = dsum_k[u];
      }
    }
  }
  if (s_fail) {
    if (threadIdx.x == 0) atomicExch(&status[5], 1);
  } else if (nstage > 0 && warp < 4) {
    // epilogue: warp w (< 4) owns TMEM lanes (= rows) 32w .. 32w+31
    const int row = warp * 32 + (threadIdx.x & 31);
    float* ps = part + (((long)blockIdx.y * gridDim.x + blockIdx.x) * 2) * (TROWS * TROWS);
    float* pk = ps + TROWS * TROWS;
    for (int which = 0; which < 2; ++which) {
      const uint32_t base = (which == 0 ? tmem_s : tmem_k) + ((uint32_t)(warp * 32) << 16);
      float* dst = which == 0 ? ps : pk;
      for (int c0 = 0; c0 < N; c0 += 16) {
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(base + (uint32_t)c0));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < valid_a) {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (c0 + j < valid_b) dst[row * TROWS + c0 + j] = __uint_as_float(r[j]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

// S, K (k x k, column-major FP64) = sums over the chunks, one warp per entry
// (lanes take every 32nd chunk, then a fixed shuffle tree).  Diagonal tiles
// are symmetrised as 0.5 (X + X^T) (as the CUDA-core path does); off-diagonal
// tiles are computed above the diagonal only and mirrored.  Diagonal entries
// come from the exact FP64 chunk sums in dpart.
__global__ void k_gram_tc_final(const float* __restrict__ part, const double* __restrict__ dpart, int nchunk,
                                int npair, const int2* __restrict__ pairs, int k, double* __restrict__ S,
                                double* __restrict__ K) {
  const int lane = threadIdx.x & 31;
  const long nwarps = (long)gridDim.x * (blockDim.x >> 5);
  const long total = (long)npair * TROWS * TROWS;
  for (long e = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < total; e += nwarps) {
    const int p = (int)(e / (TROWS * TROWS));
    const int rc = (int)(e % (TROWS * TROWS));
    const int r = rc / TROWS, c = rc % TROWS;
    const int i = pairs[p].x * TROWS + r, j = pairs[p].y * TROWS + c;
    if (i >= k || j >= k) continue;   // uniform across the warp
    const bool diag = pairs[p].x == pairs[p].y;
    const int cr = c * TROWS + r;
    double s = 0.0, kv = 0.0, st = 0.0, kt = 0.0;
    if (i == j) {
      for (int ch = lane; ch < nchunk; ch += 32) {
        s += dpart[((long)ch * 2 + 0) * k + i];
        kv += dpart[((long)ch * 2 + 1) * k + i];
      }
      s = psc_warp_sum(s);
      kv = psc_warp_sum(kv);
      if (lane == 0) {
        S[i + (long)i * k] = s;
        K[i + (long)i * k] = kv;
      }
      continue;
    }
    for (int ch = lane; ch < nchunk; ch += 32) {
      const float* ps = part + (((long)ch * npair + p) * 2) * (TROWS * TROWS);
      s += (double)ps[rc];
      kv += (double)ps[TROWS * TROWS + rc];
      if (diag) {
        st += (double)ps[cr];
        kt += (double)ps[TROWS * TROWS + cr];
      }
    }
    s = psc_warp_sum(s);
    kv = psc_warp_sum(kv);
    st = psc_warp_sum(st);
    kt = psc_warp_sum(kt);
    if (lane == 0) {
      if (diag) {
        S[i + (long)j * k] = 0.5 * (s + st);
        K[i + (long)j * k] = 0.5 * (kv + kt);
      } else {
        S[i + (long)j * k] = s;
        K[i + (long)j * k] = kv;
        S[j + (long)i * k] = s;
        K[j + (long)i * k] = kv;
      }
    }
  }
}

// Host side: returns -1 when the tensor-core path does not apply (the caller
// then uses the CUDA-core kernels).
int psc_gram_pair_tc(psc_ctx* ctx, const float* W, const float* V, long ld, int k, double* S, double* K,
                     cudaStream_t st) {
  if (!ctx->gram_tc || k < 1 || k > 512) return -1;
  const long n = ctx->n;
  const int tiles = (k + TROWS - 1) / TROWS;
  const int npair = tiles * (tiles + 1) / 2;
  // four waves of one CTA per SM by default: shorter chunks keep the FP32
  // accumulation in tensor memory short (its rounding error grows with the
  // chunk length); psc_set_gram_chunk asks for a given chunk length
  int nchunk = std::max(1, 4 * 148 / npair);
  long chunk = ((n + nchunk - 1) / nchunk + KSTAGE - 1) / KSTAGE * KSTAGE;
  if (ctx->gram_chunk > 0) chunk = (ctx->gram_chunk + KSTAGE - 1) / KSTAGE * KSTAGE;
  nchunk = (int)((n + chunk - 1) / chunk);
  const size_t tile_floats = (size_t)nchunk * npair * 2 * TROWS * TROWS;   // even, so dpart is 8-byte aligned
  PSC_REQUIRE(ctx, tile_floats * sizeof(float) <= (size_t)1 << 31,
              "gram_pair: the chunk length leaves more than 2 GiB of partial tiles");
  const size_t part_floats = tile_floats + (size_t)nchunk * 2 * k * 2;    // + nchunk x 2 x k doubles
  if (ctx->tc_part_floats < part_floats) {
    psc_dfree(ctx->tc_part);
    ctx->tc_part = nullptr;
    ctx->tc_part_floats = 0;
    PSC_CUDA(ctx, psc_dmalloc(&ctx->tc_part, part_floats * sizeof(float)));
    ctx->tc_part_floats = part_floats;
  }
  if (!ctx->tc_pairs) PSC_CUDA(ctx, psc_dmalloc(&ctx->tc_pairs, 64 * sizeof(int2)));
  if (ctx->tc_pairs_k != k) {
    int2 hp[64];
    int q = 0;
    for (int a = 0; a < tiles; ++a)
      for (int b = a; b < tiles; ++b) hp[q++] = make_int2(a, b);
    PSC_CUDA(ctx, cudaMemcpy(ctx->tc_pairs, hp, npair * sizeof(int2), cudaMemcpyHostToDevice));
    ctx->tc_pairs_k = k;
  }
  const size_t smem = 2 * (size_t)BUF_BYTES + 1024;
  PSC_CUDA(ctx, cudaFuncSetAttribute(k_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  double* dpart = reinterpret_cast<double*>(ctx->tc_part + tile_floats);
  k_gram_tc<<<dim3(npair, nchunk), TC_NT, smem, st>>>(W, V, ld, k, n, chunk, (const int2*)ctx->tc_pairs,
                                                      ctx->tc_part, dpart, ctx->wait_limit, ctx->dev_status);
  PSC_LAUNCH_CHECK(ctx);
  const long total = (long)npair * TROWS * TROWS;
  k_gram_tc_final<<<std::max(1, (int)std::min<long>(148 * 8, (total + 7) / 8)), 256, 0, st>>>(
      ctx->tc_part, dpart, nchunk, npair, (const int2*)ctx->tc_pairs, k, S, K);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_set_gram_chunk(psc_ctx* ctx, long rows) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, rows >= 0, "gram_chunk: rows < 0");
  ctx->gram_chunk = rows;
  return 0;
}

extern "C" int psc_set_gram_impl(psc_ctx* ctx, int tensor_cores) {
  if (!ctx) return 2;
  ctx->gram_tc = tensor_cores ? 1 : 0;
  return 0;
}
