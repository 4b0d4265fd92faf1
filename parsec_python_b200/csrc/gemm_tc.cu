// Tensor-core block product for the mixed-precision Rayleigh-Ritz:
// Out = W T with W an n x k FP32 block (column-major, leading dimension ld)
// and T a k x kout FP64 matrix (the R^{-1} Y of the Cholesky Rayleigh-Ritz,
// the W Q of Rayleighritz.py:4-30 / chefsi1.py:64-67), on tcgen05 with TF32
// operands split x = hi + lo and three products per term
// (hi hi + hi lo + lo hi, the dropped lo lo is ~2^-22 relative), FP32
// accumulation in tensor memory.
//
// Each CTA owns 128 grid points and every output column (up to 320: one
// accumulator of <= 256 columns, a second for the rest).  The reduction over
// the k columns of W runs in stages of 32:
//   - W's tile (128 points x 32 columns) is read with 16-byte loads that are
//     coalesced along the points, split into hi/lo in registers and stored in
//     the MN-major layout with the 128-byte / 32-byte-atom swizzle (the
//     points are the MMA's M);
//   - T's tile was split into TF32 hi/lo once per call (k_split_t) and laid
//     out as the K-major swizzled B operand, so one 1-D bulk copy per stage
//     brings it in (no tensor map, no multicast);
//   - one elected thread issues the MMAs (M = 128, N <= 256, K = 8) and
//     commits them to the stage's mbarrier.
// Two stage buffers: the loads of stage s+1 are in flight while the tensor
// cores work on stage s.  The epilogue reads TMEM with tcgen05.ld and writes
// FP32 columns, 32 consecutive points per warp store.  Every mbarrier wait is
// bounded by the context's wait limit; on a timeout the CTA records status
// word 6 and stops waiting.
//
// The FP32 accumulation rounds toward zero, which scales each output column
// by 1 - O(1e-6); consumers that need exact norms measure them (the density
// normalises each orbital by its FP64-summed norm).
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>

namespace {
constexpr int GT_NT = 256;          // 8 warps
constexpr int GT_M = 128;           // points per CTA (MMA M)
constexpr int GT_KS = 32;           // reduction columns per stage (128 bytes of FP32)
constexpr int GT_A_BYTES = GT_M * GT_KS * 4;   // 16 KB per A copy (hi or lo)
constexpr int GT_MAX_NTOT = 320;    // output columns per CTA with two stage buffers in 227 KB

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// K-major, 128-byte swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)(1024u >> 4) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;
  return d;
}

// MN-major TF32 operands take the 128-byte swizzle with 32-byte atomicity
// (layout type 1; the only MN-major layout tcgen05 accepts for 32-bit
// elements): atoms of 32 points (128 bytes) x 4 reduction rows (512 bytes),
// the 32-byte chunks of row r XOR-ed with r.  Atoms along M are 512 bytes
// apart (leading byte offset), groups of 4 reduction rows 2048 bytes apart
// (stride byte offset); one K = 8 MMA reads two groups.
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)(512u >> 4) << 16;
  d |= (uint64_t)(2048u >> 4) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)1u << 61;
  return d;
}

// kind::tf32, D F32, A TF32 MN-major, B TF32 K-major, M = 128, N
__host__ __device__ constexpr uint32_t idesc_tf32_amn(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (1u << 15) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(GT_M >> 4) << 24);
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

struct ALoad {
  float4 v[4];
};

// stage s of W: warp w loads reduction columns j = 32 s + w + 8 i (i < 4),
// lane l points p0 + 4 l .. p0 + 4 l + 3 (n and ld are multiples of 4)
__device__ __forceinline__ void a_load(const float* __restrict__ W, long ld, int k, long n, long p0, int s,
                                       ALoad& a) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const long p = p0 + 4 * l;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int j = s * GT_KS + w + 8 * i;
    float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
    if (j < k && p < n) x = __ldg(reinterpret_cast<const float4*>(W + (long)j * ld + p));
    a.v[i] = x;
  }
}

// split and store in the MN-major swizzled layout: reduction row j_local =
// w + 8 i is row kr = j_local & 3 of group g = j_local >> 2; points 4 l ..
// 4 l + 3 lie in atom l >> 3, 32-byte chunk (l & 7) >> 1 (swizzled with kr),
// half l & 1 of it
__device__ __forceinline__ void a_store(const ALoad& a, unsigned char* hi, unsigned char* lo) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float4 x = a.v[i];
    float4 h, q;
    h.x = tf32_rna(x.x); q.x = tf32_rna(x.x - h.x);
    h.y = tf32_rna(x.y); q.y = tf32_rna(x.y - h.y);
    h.z = tf32_rna(x.z); q.z = tf32_rna(x.z - h.z);
    h.w = tf32_rna(x.w); q.w = tf32_rna(x.w - h.w);
    const int jl = w + 8 * i;
    const int kr = jl & 3;
    const int off = (jl >> 2) * 2048 + (l >> 3) * 512 + kr * 128 + ((((l & 7) >> 1) ^ kr) << 5) + ((l & 1) << 4);
    *reinterpret_cast<float4*>(hi + off) = h;
    *reinterpret_cast<float4*>(lo + off) = q;
  }
}
}  // namespace

// T (k x kout, FP64, leading dimension ldt) -> per stage s: [hi | lo], each
// ntot rows (output columns, zero beyond kout) of 32 TF32 values of the
// stage's reduction rows (zero beyond k), 128-byte rows, K-major swizzle.
__global__ void k_split_t(const double* __restrict__ Tm, long ldt, int k, int kout, int ntot, int nstage,
                          float* __restrict__ out) {
  const long total = (long)nstage * ntot * GT_KS;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int kk = (int)(e % GT_KS);
    const int r = (int)((e / GT_KS) % ntot);
    const int s = (int)(e / ((long)GT_KS * ntot));
    const int j = s * GT_KS + kk;
    const double t = (j < k && r < kout) ? Tm[j + (long)r * ldt] : 0.0;
    const float f = (float)t;
    const float h = tf32_rna(f);
    const float q = tf32_rna((float)(t - (double)h));
    const long base = (long)s * 2 * ntot * GT_KS;    // floats
    const int off = r * GT_KS + ((((kk >> 2) ^ (r & 7)) << 2) | (kk & 3));
    out[base + off] = h;
    out[base + (long)ntot * GT_KS + off] = q;
  }
}

__global__ void __launch_bounds__(GT_NT, 1)
k_gemm_tc(const float* __restrict__ W, long ld, int k, long n, const float* __restrict__ Tsplit, int kout,
          int ntot, int n0, int n1, int nstage, float* __restrict__ O, long ldo, long wait_limit,
          int* status) {
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t bar_b[2];
  __shared__ __align__(8) uint64_t bar_mma[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5;
  const long p0 = (long)blockIdx.x * GT_M;
  const int b_bytes = ntot * GT_KS * 4;               // one of hi / lo
  const int buf_bytes = 2 * GT_A_BYTES + 2 * b_bytes;
  const uint32_t tmem_cols = ntot <= 32 ? 32 : ntot <= 64 ? 64 : ntot <= 128 ? 128 : ntot <= 256 ? 256 : 512;

  if (threadIdx.x == 0) {
    s_fail = 0;
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar_b[i])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar_mma[i])));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const uint32_t idesc0 = idesc_tf32_amn(n0);
  const uint32_t idesc1 = idesc_tf32_amn(n1 > 0 ? n1 : 16);

  ALoad a;
  a_load(W, ld, k, n, p0, 0, a);
  int last_commit = -1;   // thread 0: stage of the last MMA commit
  int copy_pending = -1;  // thread 0: stage whose B copy was not seen to complete
  for (int s = 0; s < nstage; ++s) {
    const int b = s & 1;
    unsigned char* buf = sm + b * buf_bytes;
    unsigned char* a_hi = buf;
    unsigned char* a_lo = buf + GT_A_BYTES;
    unsigned char* bt = buf + 2 * GT_A_BYTES;         // [hi | lo] as laid out by k_split_t
    if (s >= 2) {
      // the MMAs of stage s-2 read this buffer: wait for their commit
      if (threadIdx.x == 0 && !mbar_wait(smem_u32(&bar_mma[b]), (uint32_t)(((s - 2) >> 1) & 1), wait_limit))
        s_fail = 1;
    }
    __syncthreads();
    if (s_fail) break;
    if (threadIdx.x == 0) {
      const uint32_t bytes = 2u * (uint32_t)b_bytes;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&bar_b[b])), "r"(bytes)
                   : "memory");
      const float* src = Tsplit + (long)s * 2 * ntot * GT_KS;
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_u32(bt)),
          "l"(src), "r"(bytes), "r"(smem_u32(&bar_b[b]))
          : "memory");
      copy_pending = s;
    }
    a_store(a, a_hi, a_lo);
    if (s + 1 < nstage) a_load(W, ld, k, n, p0, s + 1, a);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      if (!mbar_wait(smem_u32(&bar_b[b]), (uint32_t)((s >> 1) & 1), wait_limit)) {
        s_fail = 1;
      } else {
        copy_pending = -1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
        const uint32_t bh = smem_u32(bt), bl = bh + (uint32_t)b_bytes;
#pragma unroll
        for (int kk = 0; kk < GT_KS / 8; ++kk) {
          const uint32_t oa = kk * 4096;   // next two groups of 4 reduction rows of the MN-major A tile
          const uint32_t ob = kk * 32;     // 8 TF32 = 32 bytes along K in the swizzled B rows
          const uint32_t acc = (s > 0 || kk > 0) ? 1u : 0u;
          mma_tf32(tmem, desc_mnmajor(ah + oa), desc_kmajor(bh + ob), idesc0, acc);
          mma_tf32(tmem, desc_mnmajor(ah + oa), desc_kmajor(bl + ob), idesc0, 1u);
          mma_tf32(tmem, desc_mnmajor(al + oa), desc_kmajor(bh + ob), idesc0, 1u);
          if (n1 > 0) {
            const uint32_t o1 = (uint32_t)n0 * 128u;   // rows n0.. of the B tile
            mma_tf32(tmem + (uint32_t)n0, desc_mnmajor(ah + oa), desc_kmajor(bh + o1 + ob), idesc1, acc);
            mma_tf32(tmem + (uint32_t)n0, desc_mnmajor(ah + oa), desc_kmajor(bl + o1 + ob), idesc1, 1u);
            mma_tf32(tmem + (uint32_t)n0, desc_mnmajor(al + oa), desc_kmajor(bh + o1 + ob), idesc1, 1u);
          }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&bar_mma[b]))
                     : "memory");
        last_commit = s;
      }
    }
  }
  if (threadIdx.x == 0) {
    // the last commit covers every MMA issued before it; after a failure,
    // one more bounded wait for the copy and the MMAs still in flight
    // before the shared and tensor memory are released
    if (last_commit >= 0) {
      const uint32_t bar = smem_u32(&bar_mma[last_commit & 1]), par = (uint32_t)((last_commit >> 1) & 1);
      if (s_fail || !mbar_wait(bar, par, wait_limit)) {
        s_fail = 1;
        mbar_wait(bar, par, PSC_DRAIN_WAIT);
      }
    }
    if (copy_pending >= 0) {
      mbar_wait(smem_u32(&bar_b[copy_pending & 1]), (uint32_t)((copy_pending >> 1) & 1), PSC_DRAIN_WAIT);
      s_fail = 1;
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (s_fail) {
    if (threadIdx.x == 0) atomicExch(&status[6], 1);
  } else if (nstage > 0) {
    // epilogue: warp w reads TMEM lanes 32 (w & 3) .. + 31 (= points), the
    // two warp groups take alternate 16-column chunks
    const int q = warp & 3;
    const long p = p0 + q * 32 + (threadIdx.x & 31);
    for (int c0 = 16 * (warp >> 2); c0 < ntot; c0 += 32) {
      uint32_t r[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (p < n) {
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (c0 + j < kout) O[p + (long)(c0 + j) * ldo] = __uint_as_float(r[j]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
}

// Host side: returns -1 when the tensor-core path does not apply (the caller
// then uses the CUDA-core kernel).  Needs 16-byte aligned W and O, n, ld and
// ldo multiples of 4, kout <= 320.
int psc_gemm_tall_tc(psc_ctx* ctx, const float* W, long ld, int k, const double* Tm, int kout, float* O, long ldo,
                     cudaStream_t st) {
  const long n = ctx->n;
  if (!ctx->gemm_tc || k < 1 || kout < 1 || (n & 3) || (ld & 3) || (ldo & 3) ||
      (reinterpret_cast<uintptr_t>(W) & 15) || (reinterpret_cast<uintptr_t>(O) & 15))
    return -1;
  int n0, n1;
  if (kout <= 256) {
    n0 = (kout + 15) & ~15;
    n1 = 0;
  } else {
    n0 = 256;
    n1 = (kout - 256 + 15) & ~15;
  }
  const int ntot = n0 + n1;
  if (ntot > GT_MAX_NTOT) return -1;
  const int nstage = (k + GT_KS - 1) / GT_KS;
  const size_t split_floats = (size_t)nstage * 2 * ntot * GT_KS;
  if (ctx->tsplit_floats < split_floats) {
    psc_dfree(ctx->tsplit);
    ctx->tsplit = nullptr;
    ctx->tsplit_floats = 0;
    PSC_CUDA(ctx, psc_dmalloc(&ctx->tsplit, split_floats * sizeof(float)));
    ctx->tsplit_floats = split_floats;
  }
  const long total = (long)nstage * ntot * GT_KS;
  k_split_t<<<std::max(1, (int)std::min<long>(592, (total + 255) / 256)), 256, 0, st>>>(Tm, k, k, kout, ntot, nstage,
                                                                                      ctx->tsplit);
  PSC_LAUNCH_CHECK(ctx);
  const size_t buf_bytes = 2 * (size_t)GT_A_BYTES + 2 * (size_t)ntot * GT_KS * 4;
  const size_t smem = 2 * buf_bytes + 1024;
  PSC_CUDA(ctx, cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_gemm_tc<<<psc_div_up(n, GT_M), GT_NT, smem, st>>>(W, ld, k, n, ctx->tsplit, kout, ntot, n0, n1, nstage, O, ldo,
                                                      ctx->wait_limit, ctx->dev_status);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_set_gemm_impl(psc_ctx* ctx, int tensor_cores) {
  if (!ctx) return 2;
  ctx->gemm_tc = tensor_cores ? 1 : 0;
  return 0;
}
