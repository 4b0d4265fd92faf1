// Forward 3-D convolution of the learned-start network on the tensor cores:
// tcgen05.mma kind::f16 with BF16 operands and FP32 accumulation in tensor
// memory, as an implicit GEMM
//   D[voxel][co] = sum_k  X[voxel][k] Wt[co][k],   k = tap * Cin + ci,
// where X is the im2col view of the virtual input (never written out: the
// upsample, the skip concatenation, the stride and the zero padding are all
// resolved while gathering) and Wt the weights transposed to [co][k].
// out[voxel][co] = act(D + bias[co]) in BF16 (and FP32 when asked).
//
// One CTA owns 128 output voxels (MMA M = 128) and all output channels (MMA
// N = Cout rounded up to 16).  The reduction runs in stages of 64 entries:
// one 128-byte row of BF16 per voxel, stored in the canonical K-major
// 128-byte-swizzled layout, so one stage is four MMAs of K = 16.  The CTA's
// threads gather stage s+1 into registers (16-byte pieces: 8 channels of one
// tap) while the MMAs of stage s run; one thread issues the MMAs and commits
// them to an mbarrier, the two-deep shared-memory ring reuses a buffer once
// its MMAs have completed.  Warps 0-3 then read the accumulators back (TMEM
// lane = voxel) and apply the bias and the activation.  Every wait is bounded
// by the context's wait limit; on a timeout the CTA drains the MMAs it issued,
// records status word 7 and writes nothing.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include "conv_geom.cuh"

namespace {
constexpr int CT_NT = 256;                  // 8 warps gather; warps 0-3 also drain tensor memory
constexpr int CT_M = 128;                   // output voxels per CTA (MMA M)
constexpr int CT_KS = 64;                   // reduction entries per stage (128 bytes of BF16)
constexpr int CT_ATILE = CT_M * 128;        // 16 KB of gathered input per stage
constexpr int CT_APER = CT_M * 8 / CT_NT;   // 16-byte input pieces per thread and stage
constexpr int CT_BPER = 256 * 8 / CT_NT;    // 16-byte weight pieces per thread and stage (N <= 256)
constexpr float CT_LEAK = 0.0625f;          // leaky-ReLU slope below zero (as the CUDA-core kernels)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
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

// instruction descriptor, kind::f16: D F32, A and B BF16, both K-major, N, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(CT_M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
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

__device__ __forceinline__ float conv_act(float a, int act) {
  return act == 1 ? fmaxf(a, 0.0f) : (act == 2 ? (a > 0.0f ? a : CT_LEAK * a) : a);
}
}  // namespace

// Wt[co][k] = W[k][co] for co < Cout and k < K, zero up to [N][Kpad]
__global__ void k_conv_wt(const __nv_bfloat16* __restrict__ W, int K, int Cout, int N, int Kpad,
                          __nv_bfloat16* __restrict__ Wt) {
  const long total = (long)N * Kpad;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int co = (int)(e / Kpad), k = (int)(e % Kpad);
    Wt[e] = (co < Cout && k < K) ? W[(long)k * Cout + co] : __float2bfloat16_rn(0.0f);
  }
}

__global__ void __launch_bounds__(CT_NT, 1)
k_conv_tc(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ S,
          const __nv_bfloat16* __restrict__ Wt, const float* __restrict__ bias, ConvGeom g, int K, int Kpad, int N,
          int act, __nv_bfloat16* __restrict__ out, float* __restrict__ out32, long wait_limit, int* status) {
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5;
  const int stage_bytes = CT_ATILE + N * 128;   // N is a multiple of 16: stages stay 1024-byte aligned
  const int ks = g.ksize, pad = ks / 2;
  const long nvo = (long)g.nxo * g.nyo * g.nzo;
  const long vo0 = (long)blockIdx.x * CT_M;
  const int nstage = Kpad / CT_KS;
  const uint32_t tcols = N <= 32 ? 32u : (N <= 64 ? 64u : (N <= 128 ? 128u : 256u));

  // this thread's pieces: rows r0 + 32 u of a stage (input rows = voxels,
  // weight rows = output channels), 16-byte piece c of each row
  const int c = threadIdx.x & 7;
  const int r0 = threadIdx.x >> 3;
  const int swz = (c ^ (r0 & 7)) << 4;   // the rows r0 + 32 u share r & 7
  int bx[CT_APER], by[CT_APER], bz[CT_APER];
  bool vok[CT_APER];
#pragma unroll
  for (int u = 0; u < CT_APER; ++u) {
    const long vo = vo0 + r0 + 32 * u;
    vok[u] = vo < nvo;
    const long v = vok[u] ? vo : 0;
    const int xo = (int)(v % g.nxo);
    const long rr = v / g.nxo;
    const int yo = (int)(rr % g.nyo), zo = (int)(rr / g.nyo);
    bx[u] = xo * g.stride - pad;
    by[u] = yo * g.stride - pad;
    bz[u] = zo * g.stride - pad;
  }

  if (threadIdx.x == 0) {
    s_fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(tcols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const uint32_t idesc = idesc_bf16(N);

  uint4 ra[CT_APER], rb[CT_BPER];
  const uint4 zero4 = make_uint4(0u, 0u, 0u, 0u);
  // the pieces of stage s: reduction entries kk .. kk+7 (one tap, 8 channels)
  auto gather = [&](int s) {
    const int kk = s * CT_KS + 8 * c;
    const bool kin = kk < K;
    const int tap = kin ? kk / g.Cin : 0;
    const int ci = kk - tap * g.Cin;
    const int dx = tap % ks, dy = (tap / ks) % ks, dz = tap / (ks * ks);
#pragma unroll
    for (int u = 0; u < CT_APER; ++u) {
      const int xi = bx[u] + dx, yi = by[u] + dy, zi = bz[u] + dz;
      const bool in = kin && vok[u] && xi >= 0 && yi >= 0 && zi >= 0 && xi < g.nxi && yi < g.nyi && zi < g.nzi;
      ra[u] = in ? conv_vin8(A, S, g, xi, yi, zi, ci) : zero4;
    }
#pragma unroll
    for (int u = 0; u < CT_BPER; ++u) {
      const int row = r0 + 32 * u;
      rb[u] = row < N ? __ldg(reinterpret_cast<const uint4*>(Wt + (long)row * Kpad + kk)) : zero4;
    }
  };

  int last_commit = -1;   // thread 0: stage of the last MMA commit
  if (nstage > 0) gather(0);
  for (int s = 0; s < nstage; ++s) {
    const int b = s & 1;
    unsigned char* abuf = sm + b * stage_bytes;
    unsigned char* bbuf = abuf + CT_ATILE;
    if (s >= 2 && threadIdx.x == 0) {
      // the MMAs of stage s-2 read this buffer: wait for their commit
      if (!mbar_wait(smem_u32(&mbar[b]), (uint32_t)(((s - 2) >> 1) & 1), wait_limit)) s_fail = 1;
    }
    __syncthreads();
    if (s_fail) break;
#pragma unroll
    for (int u = 0; u < CT_APER; ++u) *reinterpret_cast<uint4*>(abuf + (r0 + 32 * u) * 128 + swz) = ra[u];
#pragma unroll
    for (int u = 0; u < CT_BPER; ++u) {
      const int row = r0 + 32 * u;
      if (row < N) *reinterpret_cast<uint4*>(bbuf + row * 128 + swz) = rb[u];
    }
    if (s + 1 < nstage) gather(s + 1);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t aa = smem_u32(abuf), bb = smem_u32(bbuf);
#pragma unroll
      for (int kk = 0; kk < CT_KS / 16; ++kk) {
        const uint32_t o = kk * 32;   // 16 BF16 = 32 bytes along K inside the swizzled row
        mma_bf16(tmem, sw128_desc(aa + o), sw128_desc(bb + o), idesc, (s > 0 || kk > 0) ? 1u : 0u);
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
  if (s_fail) {
    if (threadIdx.x == 0) atomicExch(&status[7], 1);
  } else if (warp < 4) {
    // warp w owns tensor-memory lanes (= voxels) 32 w .. 32 w + 31
    const int row = warp * 32 + (threadIdx.x & 31);
    const long vo = vo0 + row;
    const uint32_t base = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < N; c0 += 16) {
      uint32_t r[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(base + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (vo < nvo) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int co = c0 + 8 * h;
          if (co >= g.Cout) continue;   // Cout is a multiple of 8: whole halves are in or out
          float v[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) v[j] = conv_act(__uint_as_float(r[8 * h + j]) + bias[co + j], act);
          uint4 pk;
          __nv_bfloat162* p2 = reinterpret_cast<__nv_bfloat162*>(&pk);
#pragma unroll
          for (int j = 0; j < 4; ++j) p2[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
          *reinterpret_cast<uint4*>(out + vo * g.Cout + co) = pk;
          if (out32) {
            float4* o4 = reinterpret_cast<float4*>(out32 + vo * g.Cout + co);
            o4[0] = make_float4(v[0], v[1], v[2], v[3]);
            o4[1] = make_float4(v[4], v[5], v[6], v[7]);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols));
}

// Host side of the tensor-core forward (psc_conv3d_fwd dispatches here when
// ctx->conv_tc is set); the geometry has been validated by the caller.
int psc_conv_tc_forward(psc_ctx* ctx, const ConvGeom& g, const __nv_bfloat16* a, const __nv_bfloat16* s,
                        const __nv_bfloat16* w, const float* bias, int act, __nv_bfloat16* o, float* out32,
                        cudaStream_t st) {
  const int taps = g.ksize * g.ksize * g.ksize;
  const int K = taps * g.Cin;
  const int Kpad = (K + CT_KS - 1) / CT_KS * CT_KS;
  const int N = (g.Cout + 15) / 16 * 16;
  PSC_REQUIRE(ctx, N <= 256, "conv3d: at most 256 output channels");
  PSC_REQUIRE(ctx, (reinterpret_cast<uintptr_t>(a) & 15) == 0 && (reinterpret_cast<uintptr_t>(s) & 15) == 0 &&
                       (reinterpret_cast<uintptr_t>(o) & 15) == 0 && (reinterpret_cast<uintptr_t>(out32) & 15) == 0,
              "conv3d: activations must be 16-byte aligned");
  const size_t wt_bytes = (size_t)N * Kpad * sizeof(__nv_bfloat16);
  if (ctx->conv_wt_bytes < wt_bytes) {
    psc_dfree(ctx->conv_wt);
    ctx->conv_wt = nullptr;
    ctx->conv_wt_bytes = 0;
    PSC_CUDA(ctx, psc_dmalloc(&ctx->conv_wt, wt_bytes));
    ctx->conv_wt_bytes = wt_bytes;
  }
  auto* wt = static_cast<__nv_bfloat16*>(ctx->conv_wt);
  k_conv_wt<<<std::min(148 * 4, psc_div_up((long)N * Kpad, 256)), 256, 0, st>>>(w, K, g.Cout, N, Kpad, wt);
  PSC_LAUNCH_CHECK(ctx);
  const size_t smem = 2 * (size_t)(CT_ATILE + N * 128) + 1024;
  PSC_CUDA(ctx, cudaFuncSetAttribute(k_conv_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long nvo = (long)g.nxo * g.nyo * g.nzo;
  k_conv_tc<<<psc_div_up(nvo, CT_M), CT_NT, smem, st>>>(a, s, wt, bias, g, K, Kpad, N, act, o, out32,
                                                       ctx->wait_limit, ctx->dev_status);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_set_conv_impl(psc_ctx* ctx, int impl) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, impl >= 0 && impl <= 2, "conv_impl: 0 (CUDA cores), 1 (by layer) or 2 (tensor cores)");
  ctx->conv_tc = impl;
  return 0;
}
