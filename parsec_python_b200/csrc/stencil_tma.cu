// TMA-fed stencil pipeline (sm_100a): the fused Chebyshev / H.X step
//   Out = a * (W In) + b * In + g * Prev,  W = c0 + sum_d c_d (shifts) [+ diag(pot)]
// with plane windows streamed into shared memory by 1-D bulk copies.
//
// A CTA owns S = 512 consecutive flat xy points of one column and a chunk of
// z planes.  For every plane the points it needs -- its own S points plus R
// rows of y halo on each side -- are one contiguous range of the plane, so a
// single cp.async.bulk (no tensor map, no multicast) moves it into a slot of
// a ring of NBUF = R + 1 + D shared-memory windows, completing on the slot's
// mbarrier.  The z neighbours of each point live in a register queue fed from
// the ring; x and y neighbours are read from the current plane's window with
// 16-byte loads (each thread owns two adjacent x points; the pair itself comes
// from the queue).  Prev and pot are read straight from global memory one
// plane ahead, so they cost no shared-memory traffic.  D planes are in flight
// per CTA at all times, which is what keeps HBM busy.
//
// Every mbarrier wait is bounded: on timeout the CTA records the failure in
// status[3] and carries on without waiting (results are then garbage but the
// GPU is never hung).  Every bulk copy issued is waited for before the CTA
// exits.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <cstdint>

namespace {

constexpr int TNT = 256;          // threads per CTA
constexpr int TS = 2 * TNT;       // points per slab (two per thread)
constexpr int TD = 2;             // planes prefetched beyond the one consumed next
constexpr long WAIT_LIMIT = 1L << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait; returns false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long i = 0; i < WAIT_LIMIT; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
  using type = double2;
};
template <>
struct Vec2<float> {
  using type = float2;
};

template <typename T>
struct TmaArgs {
  const T* X;
  long ldx;
  const T* P;
  long ldp;
  T* Y;
  long ldy;
  const T* pot;
  int nx, ny, nz, zchunk;
  T c0, c[4];
  const double* coef;
  double a, b, g;
  int* status;
};

}  // namespace

template <typename T, int R>
__global__ void __launch_bounds__(TNT)
k_stencil_tma(TmaArgs<T> A) {
  using V2 = typename Vec2<T>::type;
  constexpr int NBUF = R + 1 + TD;   // X plane windows resident
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nx = A.nx, ny = A.ny, nz = A.nz;
  const int nxy = nx * ny;
  const int H = R * nx;
  const int WIN = TS + 2 * H;
  T* ring = reinterpret_cast<T*>(smem_raw);                 // [NBUF][WIN]
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + (size_t)NBUF * WIN);  // [NBUF]
  __shared__ int s_fail;

  const int slab0 = blockIdx.x * TS;
  const int z0 = blockIdx.y * A.zchunk;
  const int z1 = min(nz, z0 + A.zchunk);
  const int zlast = min(nz, z1 + R);  // X planes needed: [z0 - R, z1 + R) within [0, nz)
  const long col = blockIdx.z;
  const T* Xc = A.X + col * A.ldx;
  const T* Pc = A.P ? A.P + col * A.ldp : nullptr;
  T* Yc = A.Y + col * A.ldy;
  const bool has_pot = A.pot != nullptr;

  T ca, cb, cg;
  if (A.coef) { ca = (T)A.coef[0]; cb = (T)A.coef[1]; cg = (T)A.coef[2]; }
  else { ca = (T)A.a; cb = (T)A.b; cg = (T)A.g; }

  // valid part of the window within the plane
  const int w0 = slab0 - H;
  const int v0 = max(0, w0), v1 = min(nxy, slab0 + TS + H);
  const uint32_t xbytes = (uint32_t)((v1 - v0) * sizeof(T));
  const int seff = min(TS, nxy - slab0);

  // zero the parts of every window that lie outside the plane (never written by the copies)
  for (int s = 0; s < NBUF; ++s) {
    T* w = ring + (size_t)s * WIN;
    for (int i = threadIdx.x; i < WIN; i += TNT) {
      const int f = w0 + i;
      if (f < v0 || f >= v1) w[i] = T(0);
    }
  }
  if (threadIdx.x == 0) {
    s_fail = 0;
    for (int i = 0; i < NBUF; ++i) mbar_init(&bars[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();

  auto issue_x = [&](int p) {  // plane p into slot (p - z0) mod NBUF; only z0 <= p < zlast
    const int s = (p - z0) % NBUF;
    uint64_t* bar = &bars[s];
    mbar_expect_tx(bar, xbytes);
    bulk_g2s(ring + (size_t)s * WIN + (v0 - w0), Xc + (long)p * nxy + v0, xbytes, bar);
  };
  if (threadIdx.x == 0) {
    for (int p = z0; p < min(zlast, z0 + NBUF); ++p) issue_x(p);
  }

  // own pair of points
  const int loc = 2 * threadIdx.x;
  const bool own = loc < seff;
  const int q = slab0 + loc;
  const int xi = own ? q % nx : 0;
  const int s_c = H + loc;  // window offset of the pair

  // Prev and pot of the pair, one plane ahead in registers (P may alias Y:
  // a point of P is read before this thread overwrites it)
  V2 pv_next{T(0), T(0)}, po_next{T(0), T(0)};
  auto load_pp = [&](int z) {
    if (!own || z >= z1) return;
    if (Pc) pv_next = *reinterpret_cast<const V2*>(Pc + (long)z * nxy + q);
    if (has_pot) po_next = *reinterpret_cast<const V2*>(A.pot + (long)z * nxy + q);
  };
  load_pp(z0);

  // z queue from direct loads of the planes below the chunk
  T zq0[2 * R + 1], zq1[2 * R + 1];
#pragma unroll
  for (int i = 0; i < 2 * R; ++i) {
    const int zz = z0 - R + i;
    zq0[i] = zq1[i] = T(0);
    if (zz < z0) {
      if (own && zz >= 0) {
        const V2 v = *reinterpret_cast<const V2*>(Xc + (long)zz * nxy + q);
        zq0[i] = v.x;
        zq1[i] = v.y;
      }
    }
  }
  bool fail = false;
  // planes z0 .. z0+R-1 enter the queue from the ring
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int p = z0 + i;
    if (p < nz) {
      const int s = (p - z0) % NBUF;
      if (!fail && !mbar_wait(&bars[s], ((p - z0) / NBUF) & 1)) fail = true;
      if (own) {
        const V2 v = *reinterpret_cast<const V2*>(ring + (size_t)s * WIN + s_c);
        zq0[R + i] = v.x;
        zq1[R + i] = v.y;
      }
    }
  }

  // per-thread x-boundary weights: a neighbour across the row edge gets 0
  T cl0[R], cr0[R], cl1[R], cr1[R];
#pragma unroll
  for (int d = 1; d <= R; ++d) {
    const T cd = A.c[d - 1];
    cl0[d - 1] = (xi - d >= 0) ? cd : T(0);
    cr0[d - 1] = (xi + d < nx) ? cd : T(0);
    cl1[d - 1] = (xi + 1 - d >= 0) ? cd : T(0);
    cr1[d - 1] = (xi + 1 + d < nx) ? cd : T(0);
  }
  const T c0 = A.c0;
  // z loop unrolled by Q = 2R+1 so the register queue rotates by renaming:
  // at unrolled position u, plane z - R + i lives in zq[(u + i) % Q]
  constexpr int Q = 2 * R + 1;
#pragma unroll 1
  for (int zb = z0; zb < z1; zb += Q) {
#pragma unroll
    for (int u = 0; u < Q; ++u) {
      const int z = zb + u;
      if (z >= z1) break;
      // queue front: plane z + R
      const int pf = z + R;
      T f0 = T(0), f1 = T(0);
      if (pf < nz) {
        const int s = (pf - z0) % NBUF;
        if (!fail && !mbar_wait(&bars[s], ((pf - z0) / NBUF) & 1)) fail = true;
        if (own) {
          const V2 v = *reinterpret_cast<const V2*>(ring + (size_t)s * WIN + s_c);
          f0 = v.x;
          f1 = v.y;
        }
      }
      zq0[(u + 2 * R) % Q] = f0;
      zq1[(u + 2 * R) % Q] = f1;
      const V2 pvv = pv_next, pov = po_next;
      load_pp(z + 1);
      const T* pl = ring + (size_t)((z - z0) % NBUF) * WIN;
      if (own) {
        // x neighbours: window values s_c - R .. s_c + R + 1, fetched as aligned
        // pairs starting at the even offset s_c - R - (R & 1); the pair itself
        // (pair index CJ) is the queue's centre
        constexpr int NP = R + 1 + (R & 1);
        constexpr int OFF = R + (R & 1);  // xs index of the pair's first point
        constexpr int CJ = OFF / 2;
        const T xc0 = zq0[(u + R) % Q], xc1 = zq1[(u + R) % Q];
        T xs[2 * NP];
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          if (j == CJ) {
            xs[2 * j] = xc0;
            xs[2 * j + 1] = xc1;
          } else {
            const V2 v = *reinterpret_cast<const V2*>(pl + s_c - R - (R & 1) + 2 * j);
            xs[2 * j] = v.x;
            xs[2 * j + 1] = v.y;
          }
        }
        // two partial sums per point: y + z terms, x terms
        T acc0 = c0 * xc0, acc1 = c0 * xc1;
        T ax0 = T(0), ax1 = T(0);
#pragma unroll
        for (int d = 1; d <= R; ++d) {
          // rows outside the plane are zero in the window, so y needs no test
          const V2 ym = *reinterpret_cast<const V2*>(pl + s_c - d * nx);
          const V2 yp = *reinterpret_cast<const V2*>(pl + s_c + d * nx);
          const T cd = A.c[d - 1];
          const T t0 = (ym.x + yp.x) + (zq0[(u + R - d) % Q] + zq0[(u + R + d) % Q]);
          const T t1 = (ym.y + yp.y) + (zq1[(u + R - d) % Q] + zq1[(u + R + d) % Q]);
          acc0 += cd * t0;
          acc1 += cd * t1;
          ax0 += cl0[d - 1] * xs[OFF - d];
          ax0 += cr0[d - 1] * xs[OFF + d];
          ax1 += cl1[d - 1] * xs[OFF + 1 - d];
          ax1 += cr1[d - 1] * xs[OFF + 1 + d];
        }
        acc0 += ax0;
        acc1 += ax1;
        if (has_pot) {
          acc0 += pov.x * xc0;
          acc1 += pov.y * xc1;
        }
        T o0 = ca * acc0 + cb * xc0;
        T o1 = ca * acc1 + cb * xc1;
        if (Pc) {
          o0 += cg * pvv.x;
          o1 += cg * pvv.y;
        }
        V2 o;
        o.x = o0;
        o.y = o1;
        *reinterpret_cast<V2*>(Yc + (long)z * nxy + q) = o;
      }
      __syncthreads();  // slot of plane z is free
      if (threadIdx.x == 0) {
        const int pn = z + NBUF;
        if (pn < zlast) issue_x(pn);
      }
    }
  }
  if (fail) s_fail = 1;
  __syncthreads();
  if (threadIdx.x == 0 && s_fail) atomicExch(&A.status[3], 1);
}

// Alignment rules of the 1-D bulk copies: 16-byte aligned addresses and
// sizes, i.e. even (FP64) or multiple-of-4 (FP32) element offsets.
template <typename T>
static bool tma_ok(const psc_ctx* ctx, const void* X, long ldx, const void* P, long ldp, const void* Y, long ldy) {
  const long q = 16 / sizeof(T);
  const long nxy = (long)ctx->nx * ctx->ny;
  if (nxy % q || (ctx->radius * (long)ctx->nx) % q || ldx % q || (P && ldp % q) || ldy % q) return false;
  if (ctx->nx % 2) return false;  // pairs must not straddle rows
  if (((uintptr_t)X | (uintptr_t)Y | (uintptr_t)P) % 16) return false;
  return true;
}

template <typename T, int R>
static int launch_tma_t(psc_ctx* ctx, int k, const T* X, long ldx, const T* P, long ldp, T* Y, long ldy,
                        const T* pot, const double* w, const double* coef, double a, double b, double g,
                        cudaStream_t st) {
  const int nxy = ctx->nx * ctx->ny;
  const int nslab = (nxy + TS - 1) / TS;
  // z chunks: enough CTAs for ~8 waves of 2 CTAs per SM, chunks of >= 8 planes
  const long want = 148L * 2 * 8;
  long per_col = (want + k - 1) / k;
  int nzc = (int)std::max<long>(1, std::min<long>(ctx->nz, (per_col + nslab - 1) / nslab));
  int zchunk = (ctx->nz + nzc - 1) / nzc;
  const int zmin = std::min(ctx->nz, 8);
  if (zchunk < zmin) zchunk = zmin;
  nzc = (ctx->nz + zchunk - 1) / zchunk;
  constexpr int NBUF = R + 1 + TD;
  const size_t win = TS + 2 * (size_t)R * ctx->nx;
  const size_t smem = NBUF * win * sizeof(T) + NBUF * sizeof(uint64_t);
  if (smem > 220 * 1024) return -1;  // window too wide: the register-queue kernel takes it
  auto kern = k_stencil_tma<T, R>;
  PSC_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  TmaArgs<T> A;
  A.X = X; A.ldx = ldx; A.P = P; A.ldp = ldp; A.Y = Y; A.ldy = ldy; A.pot = pot;
  A.nx = ctx->nx; A.ny = ctx->ny; A.nz = ctx->nz; A.zchunk = zchunk;
  A.c0 = (T)w[0];
  for (int i = 0; i < 4; ++i) A.c[i] = (T)w[1 + i];
  A.coef = coef; A.a = a; A.b = b; A.g = g; A.status = ctx->dev_status;
  kern<<<dim3(nslab, nzc, k), TNT, smem, st>>>(A);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

// Returns -1 if the TMA path does not apply (caller uses the register kernel).
template <typename T>
int psc_stencil_tma(psc_ctx* ctx, int k, const T* X, long ldx, const T* P, long ldp, T* Y, long ldy, const T* pot,
                    const double* w, const double* coef, double a, double b, double g, cudaStream_t st) {
  if (!tma_ok<T>(ctx, X, ldx, P, ldp, Y, ldy)) return -1;
  switch (ctx->radius) {
    case 1: return launch_tma_t<T, 1>(ctx, k, X, ldx, P, ldp, Y, ldy, pot, w, coef, a, b, g, st);
    case 2: return launch_tma_t<T, 2>(ctx, k, X, ldx, P, ldp, Y, ldy, pot, w, coef, a, b, g, st);
    case 3: return launch_tma_t<T, 3>(ctx, k, X, ldx, P, ldp, Y, ldy, pot, w, coef, a, b, g, st);
    case 4: return launch_tma_t<T, 4>(ctx, k, X, ldx, P, ldp, Y, ldy, pot, w, coef, a, b, g, st);
  }
  return -1;
}

template int psc_stencil_tma<double>(psc_ctx*, int, const double*, long, const double*, long, double*, long,
                                     const double*, const double*, const double*, double, double, double,
                                     cudaStream_t);
template int psc_stencil_tma<float>(psc_ctx*, int, const float*, long, const float*, long, float*, long,
                                    const float*, const double*, const double*, double, double, double,
                                    cudaStream_t);
