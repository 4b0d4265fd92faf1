// TMA-fed stencil pipeline (sm_100a): the fused Chebyshev / H.X step
//   Out = a * (W In) + b * In + g * Prev,  W = c0 + sum_d c_d (shifts) [+ diag(pot)]
// with plane windows streamed into shared memory by 1-D bulk copies.
//
// A CTA owns S = 512 (FP64) or 1024 (FP32) consecutive flat xy points of one
// column and a chunk of z planes.  For every plane the points it needs -- its
// own S points plus R rows of y halo on each side -- are one contiguous range
// of the plane, so a single cp.async.bulk (no tensor map, no multicast) moves
// it into a slot of a ring of NBUF = R + 1 + D shared-memory windows (D = 3),
// completing on the slot's mbarrier.  Each slot ends with one zero vector.
// The z neighbours of each point live in a register queue fed from the ring;
// x and y neighbours are read from the current plane's window with 16-byte
// loads (each thread owns a run of 2 FP64 or 4 FP32 points).  When the run
// cannot cross a row edge (2 | nx for FP64, 4 | nx for FP32) the x vectors
// outside the row are read from the zero vector, so the x terms need no
// per-point masks; otherwise each point masks its x neighbours by its
// distances to the row edges.  Prev and pot are prefetched three planes ahead
// by per-thread 16-byte cp.async copies into a small shared-memory ring that
// each thread reads back itself (no block-wide handshake).  D planes of X are
// in flight per CTA at all times, which is what keeps HBM busy.
//
// Every mbarrier wait is bounded by the context's wait limit: on timeout the
// CTA records the failure in status[3], stops issuing copies and carries on
// without waiting (results are then garbage but the GPU is never hung).
// Every bulk copy issued is waited for before the CTA exits.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <queue>
#include <type_traits>
#include <vector>

namespace {

#ifndef PSC_STENCIL_THREADS
#define PSC_STENCIL_THREADS 256
#endif
constexpr int TNT = PSC_STENCIL_THREADS;  // threads per CTA
#ifndef PSC_STENCIL_CTAS_PER_SM
#define PSC_STENCIL_CTAS_PER_SM 2   // resident CTAs per SM (registers and shared memory)
#endif
// planes of X prefetched beyond the one consumed next
#ifndef PSC_STENCIL_PREFETCH_F64
#define PSC_STENCIL_PREFETCH_F64 3
#endif
#ifndef PSC_STENCIL_PREFETCH_F32
#define PSC_STENCIL_PREFETCH_F32 3
#endif
#ifndef PSC_STENCIL_PP_SLOTS
#define PSC_STENCIL_PP_SLOTS 4
#endif
template <typename T>
__host__ __device__ constexpr int prefetch_depth() {
  return sizeof(T) == 8 ? PSC_STENCIL_PREFETCH_F64 : PSC_STENCIL_PREFETCH_F32;
}
constexpr int PP_SLOTS = PSC_STENCIL_PP_SLOTS;  // Prev/pot slots: the plane in use + the prefetched
#ifndef PSC_STENCIL_SYNC_EVERY
#define PSC_STENCIL_SYNC_EVERY 2
#endif
constexpr int SYNC_EVERY = PSC_STENCIL_SYNC_EVERY;  // planes between block barriers

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
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long limit) {
  for (long i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Points per thread: 16-byte vectors (two FP64 or four FP32 points), or
// 8-byte vectors of two FP32 points when nx is only even (the runs then never
// cross a row, so the x terms need no per-point masks).
template <typename T, int VW>
struct VecOf;
template <>
struct VecOf<double, 2> {
  using type = double2;
};
template <>
struct VecOf<float, 4> {
  using type = float4;
};
template <>
struct VecOf<float, 2> {
  using type = float2;
};

template <int VW, typename T>
__device__ __forceinline__ void vload(const T* p, T* out) {
  using V = typename VecOf<T, VW>::type;
  const V v = *reinterpret_cast<const V*>(p);
  const T* e = reinterpret_cast<const T*>(&v);
#pragma unroll
  for (int j = 0; j < VW; ++j) out[j] = e[j];
}

template <int VW, typename T>
__device__ __forceinline__ void vstore(T* p, const T* in) {
  using V = typename VecOf<T, VW>::type;
  V v;
  T* e = reinterpret_cast<T*>(&v);
#pragma unroll
  for (int j = 0; j < VW; ++j) e[j] = in[j];
  *reinterpret_cast<V*>(p) = v;
}

// load VW consecutive values from an address aligned to A elements (A | VW)
template <typename T, int A, int VW>
__device__ __forceinline__ void vload_a(const T* p, T* out) {
  if constexpr (A == VW) {
    vload<VW>(p, out);
  } else if constexpr (A == 2) {
    using V2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
#pragma unroll
    for (int h = 0; h < VW / 2; ++h) {
      const V2 v = *reinterpret_cast<const V2*>(p + 2 * h);
      out[2 * h] = v.x;
      out[2 * h + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int j = 0; j < VW; ++j) out[j] = p[j];
  }
}

// The y row at distance d from the run: the window offset of the run is a
// multiple of VW plus R nx, and R nx is a multiple of VW (a condition of the
// TMA path), so the row starts d nx away from a VW-aligned spot and is
// aligned to min(VW, YA 2^v) elements, 2^v the power of two in d (YA holds
// nx's).  d is a constant after unrolling, so the choice folds away.
template <typename T, int YA, int VW>
__device__ __forceinline__ void vload_row(const T* p, int d, T* out) {
  int a = YA;
  while (a < VW && (d & 1) == 0) {
    a *= 2;
    d >>= 1;
  }
  if (a >= VW)
    vload<VW>(p, out);
  else if (a >= 2)
    vload_a<T, 2, VW>(p, out);
  else
    vload_a<T, 1, VW>(p, out);
}

// per-thread asynchronous copy of one run (VW points) into shared memory
template <int BYTES>
__device__ __forceinline__ void cp_async_run(void* dst, const void* src) {
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

template <int VW>
__host__ __device__ constexpr int slab_points() {
  return VW * TNT;
}

template <typename T>
struct TmaArgs {
  const T* X;
  long ldx;
  const T* P;
  long ldp;
  T* Y;
  long ldy;
  const T* pot;
  int nx, ny, nz;
  const int4* sched;  // per CTA: column, slab, first plane, end plane
  T c0, c[4];
  T csr;              // FP32 weights: minus their sum-rule residual, (c0 + 6 sum_d c_d) in FP32 - in FP64
  const double* coef;
  double a, b, g;
  long wait_limit;    // polls of each mbarrier wait before the CTA gives up
  // sphere mask: outputs at points with (i h - cx)^2 + (j h - cy)^2 +
  // (l h - cz)^2 > mask_r2 are zero (mask_r2 = 0: the whole cube)
  double mask_r2, h, cx, cy, cz;
  int* status;
};

}  // namespace

// YA: alignment (in elements) of the y-neighbour rows, the largest of VW, 2, 1
// that divides nx; their loads are split to match.  MODE (FP32 only):
// bit 0 = the arithmetic on packed pairs of points, bit 1 = sum-rule
// correction: with the weights rounded to FP32 the sum rule c0 + 6 sum_d c_d
// = 0 fails by their rounding errors (-6.1e-8 Ha at h = 0.47 bohr), a
// constant shift of every eigenvalue that the band energy multiplies by the
// electron count; one more term, -(that residual) x, removes it.  (Applying
// every weight as its FP32 value plus its rounding error moved the
// Rayleigh quotients of smooth fields by no more than this one term does.)
template <typename T, int R, int YA, int VW, int MODE>
__global__ void __launch_bounds__(TNT)
k_stencil_tma(TmaArgs<T> A) {
  constexpr bool PK = (MODE & 1) != 0;
  constexpr bool COMP = (MODE & 2) != 0;
  static_assert(!PK || (sizeof(T) == 4 && VW % 2 == 0), "packed pairs need FP32 runs of an even length");
  static_assert(!COMP || sizeof(T) == 4, "compensated weights are for FP32");
  constexpr int TS = slab_points<VW>();    // points per slab (VW per thread)
  constexpr int NBUF = R + 1 + prefetch_depth<T>();   // X plane windows resident
  constexpr int NS = PP_SLOTS;
  constexpr int Q = 2 * R + 1;             // z queue length
  static_assert(SYNC_EVERY >= 1 && SYNC_EVERY <= NBUF - R, "barrier interval exceeds the ring");
  constexpr int HV = (R + VW - 1) / VW;    // x-halo vectors on each side
  constexpr int NPV = 2 * HV + 1;          // x vectors per row (the centre one comes from the queue)
  constexpr int OFF = HV * VW;             // xs index of the thread's first point
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nx = A.nx, ny = A.ny, nz = A.nz;
  const int nxy = nx * ny;
  const int H = R * nx;
  const int WIN = TS + 2 * H;
  // slot stride: the window and one zero vector, rounded up to 16 bytes so
  // that every slot starts where a bulk copy may write
  constexpr int Q16 = 16 / (int)sizeof(T);
  const int WS = (WIN + VW + Q16 - 1) / Q16 * Q16;
  T* ring = reinterpret_cast<T*>(smem_raw);                                   // [NBUF][WS]
  T* pring = ring + (size_t)NBUF * WS;                                        // [NS][2][TS]: Prev, pot
  uint64_t* bars = reinterpret_cast<uint64_t*>(pring + (size_t)NS * 2 * TS);  // [NBUF]
  __shared__ int s_fail;

  const int4 work = A.sched[blockIdx.x];
  const int slab0 = work.y * TS;
  const int z0 = work.z;
  const int z1 = work.w;
  if (work.x < 0) {
    // sphere mask: planes of this slab that hold no point inside the sphere;
    // the output is zero there and nothing is read
    const int loc0 = VW * threadIdx.x;
    if (loc0 < min(TS, nxy - slab0)) {
      T zv[VW];
#pragma unroll
      for (int j = 0; j < VW; ++j) zv[j] = T(0);
      T* Yz = A.Y + (long)(-1 - work.x) * A.ldy + slab0 + loc0;
      for (int z = z0; z < z1; ++z) vstore<VW>(Yz + (long)z * nxy, zv);
    }
    return;
  }
  const int zlast = min(nz, z1 + R);  // X planes needed: [z0 - R, z1 + R) within [0, nz)
  const long col = work.x;
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

  // zero the parts of every window that lie outside the plane and the pad
  // vector after it (neither is ever written by the copies)
  for (int s = 0; s < NBUF; ++s) {
    T* w = ring + (size_t)s * WS;
    for (int i = threadIdx.x; i < WS; i += TNT) {
      const int f = w0 + i;
      if (i >= WIN || f < v0 || f >= v1) w[i] = T(0);
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
    bulk_g2s(ring + (size_t)s * WS + (v0 - w0), Xc + (long)p * nxy + v0, xbytes, bar);
  };
  int issued = min(zlast, z0 + NBUF);  // next plane to copy (thread 0's count)
  if (threadIdx.x == 0) {
    for (int p = z0; p < issued; ++p) issue_x(p);
  }

  // own run of VW points (it may cross a row boundary: every point has its own x)
  const int loc = VW * threadIdx.x;
  const bool own = loc < seff;
  const int q = slab0 + loc;
  const int s_c = H + loc;  // window offset of the run

  // Prev and pot of the run, NS-1 planes ahead: each thread copies its own
  // 16-byte run with cp.async into slot (z - z0) mod NS and reads it back
  // itself, so no block-wide handshake is needed.  One commit group per
  // plane (empty ones too), so "wait until at most NS-2 groups are pending"
  // means plane z has landed.  (P may alias Y: plane z of P is read before
  // this thread stores plane z of Y.)
  const bool use_pp = Pc || has_pot;
  auto copy_pp = [&](int z) {
    if (own && z < z1) {
      T* d = pring + (size_t)((z - z0) % NS) * 2 * TS + loc;
      if (Pc) cp_async_run<VW * sizeof(T)>(d, Pc + (long)z * nxy + q);
      if (has_pot) cp_async_run<VW * sizeof(T)>(d + TS, A.pot + (long)z * nxy + q);
    }
    cp_async_commit();
  };
  if (use_pp)
    for (int z = z0; z < z0 + NS - 1; ++z) copy_pp(z);

  // z queue: planes below the chunk from global memory, z0 .. z0+R-1 from the ring
  T zq[VW][Q];
#pragma unroll
  for (int i = 0; i < 2 * R; ++i) {
    const int zz = z0 - R + i;
#pragma unroll
    for (int j = 0; j < VW; ++j) zq[j][i] = T(0);
    if (zz < z0 && own && zz >= 0) {
      T v[VW];
      vload<VW>(Xc + (long)zz * nxy + q, v);
#pragma unroll
      for (int j = 0; j < VW; ++j) zq[j][i] = v[j];
    }
  }
  bool fail = false;
  int fail_plane = zlast;   // first plane whose wait this thread gave up on
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int p = z0 + i;
    if (p < nz) {
      const int s = (p - z0) % NBUF;
      if (!fail && !mbar_wait(&bars[s], ((p - z0) / NBUF) & 1, A.wait_limit)) {
        fail = true;
        fail_plane = p;
      }
      if (own) {
        T v[VW];
        vload<VW>(ring + (size_t)s * WS + s_c, v);
#pragma unroll
        for (int j = 0; j < VW; ++j) zq[j][R + i] = v[j];
      }
    }
  }

  // When VW divides nx, a thread's run lies in one row and every aligned
  // x vector around it is either wholly in that row or wholly outside it:
  // the outside ones are read from the slot's zero pad, so the x terms need
  // no per-point masks.  Otherwise (FP32 runs crossing a row edge) each point
  // keeps its distances to the row edges, capped at R: a neighbour d > el
  // (left) or d > er (right) lies across the edge and gets weight 0.
  constexpr bool EXACT = (YA == VW);
  int xo[NPV];
#pragma unroll
  for (int v = 0; v < NPV; ++v) {
    const int xv = (own ? q % nx : 0) - OFF + v * VW;  // first x of vector v
    xo[v] = (xv >= 0 && xv + VW <= nx) ? s_c - OFF + v * VW : WIN;
  }
  int el[VW], er[VW];
#pragma unroll
  for (int j = 0; j < VW; ++j) {
    const int xj = own ? (q + j) % nx : 0;
    el[j] = min(R, xj);
    er[j] = min(R, nx - 1 - xj);
  }
  // Pair masks (FP32 4-point runs with packed arithmetic, nx = 2 mod 4):
  // the run's 12-value x window is six aligned pairs, none of which crosses
  // a row (nx is even), and the run itself splits into two pairs, A (points
  // 0, 1) and B (points 2, 3), each in one row.  A window pair is a valid x
  // neighbour of A's points iff it lies in A's row, likewise for B, so the
  // edge masks are twelve loop-invariant 0/1 factors (instead of a compare
  // and a select per point and distance in every plane).  mA[p], mB[p]:
  // pair p of the window (flat q - 4 + 2p) for owner A, B.
  constexpr bool PAIRM = (YA != VW) && PK && VW == 4 && YA == 2 && R <= 4;
  float mA[6], mB[6];
  if constexpr (PAIRM) {
    const int x0 = own ? q % nx : 0;
    const bool b_next = x0 + 2 > nx - 2;   // B starts the next row
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      const int xp = x0 - 4 + 2 * p;       // x of the pair's first point, in A's row coordinates
      mA[p] = (xp >= 0 && xp <= nx - 2) ? 1.f : 0.f;
      mB[p] = b_next ? (xp >= nx ? 1.f : 0.f) : mA[p];
    }
  }
  const bool masked = A.mask_r2 > 0.0;
  double mxy[VW];   // (x^2 + y^2) of the run's points, for the sphere mask
#pragma unroll
  for (int j = 0; j < VW; ++j) {
    const int qq = own ? q + j : 0;
    const double xm = (qq % nx) * A.h - A.cx, ym = (qq / nx) * A.h - A.cy;
    mxy[j] = xm * xm + ym * ym;
  }
  const T c0 = A.c0;
  // z loop unrolled by Q so the register queue rotates by renaming:
  // at unrolled position u, plane z - R + i lives in zq[.][(u + i) % Q]
#pragma unroll 1
  for (int zb = z0; zb < z1; zb += Q) {
#pragma unroll
    for (int u = 0; u < Q; ++u) {
      const int z = zb + u;
      if (z >= z1) break;
      // queue front: plane z + R
      const int pf = z + R;
      {
        T f[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) f[j] = T(0);
        if (pf < nz) {
          const int s = (pf - z0) % NBUF;
          if (!fail && !mbar_wait(&bars[s], ((pf - z0) / NBUF) & 1, A.wait_limit)) {
            fail = true;
            fail_plane = pf;
          }
          if (own) vload<VW>(ring + (size_t)s * WS + s_c, f);
        }
#pragma unroll
        for (int j = 0; j < VW; ++j) zq[j][(u + 2 * R) % Q] = f[j];
      }
      T pvv[VW], pov[VW];
#pragma unroll
      for (int j = 0; j < VW; ++j) pvv[j] = pov[j] = T(0);
      if (use_pp) {
        copy_pp(z + NS - 1);
        cp_async_wait<NS - 1>();
        if (own) {
          const T* pp = pring + (size_t)((z - z0) % NS) * 2 * TS + loc;
          if (Pc) vload<VW>(pp, pvv);
          if (has_pot) vload<VW>(pp + TS, pov);
        }
      }
      const T* pl = ring + (size_t)((z - z0) % NBUF) * WS;
      if (own) {
        // x neighbours: the aligned vectors around the run (the run itself is
        // the queue's centre).  Row-aligned runs (EXACT) read the vectors
        // outside the row from the slot's zero pad; otherwise each point
        // masks its neighbours by its distances to the row edges.
        T xs[NPV * VW];
#pragma unroll
        for (int v = 0; v < NPV; ++v) {
          if (v == HV) {
#pragma unroll
            for (int j = 0; j < VW; ++j) xs[v * VW + j] = zq[j][(u + R) % Q];
          } else {
            vload<VW>(pl + (EXACT ? xo[v] : s_c - OFF + v * VW), xs + v * VW);
          }
        }
        auto xl = [&](int j, int d) -> T { return (EXACT || d <= el[j]) ? xs[OFF + j - d] : T(0); };
        auto xr = [&](int j, int d) -> T { return (EXACT || d <= er[j]) ? xs[OFF + j + d] : T(0); };
        // per point: acc = c0 x + sum_d c_d (((y-d + y+d) + (z-d + z+d)) + (x-d + x+d)),
        // and with compensated weights the same sum over the weights'
        // rounding errors in its own (small) accumulator.  FP32 sums the
        // shells from d = R down to 1 and adds c0 x last: of the orders
        // tried this leaves the smallest bias in the Rayleigh quotients of
        // smooth fields (the low spectrum), about 3e-9 Ha.
        constexpr bool REV = sizeof(T) == 4;
        T o[VW];
        if constexpr (PK) {
          constexpr int NP = VW / 2;
          // the window masked for each owner pair (PAIRM): 16 multiplies
          float xa[PAIRM ? NPV * VW : 1], xb[PAIRM ? NPV * VW : 1];
          if constexpr (PAIRM) {
#pragma unroll
            for (int i = 0; i < NPV * VW; ++i) {
              const int p = i >> 1;
              xa[i] = p == 2 ? xs[i] : xs[i] * mA[p];
              xb[i] = p == 3 ? xs[i] : xs[i] * mB[p];
            }
          }
          float2 acc[NP];
#pragma unroll
          for (int h = 0; h < NP; ++h) {
            const float2 xc = make_float2(xs[OFF + 2 * h], xs[OFF + 2 * h + 1]);
            acc[h] = REV ? make_float2(0.f, 0.f) : __fmul2_rn(make_float2(c0, c0), xc);
          }
#pragma unroll
          for (int dd = 0; dd < R; ++dd) {
            const int d = REV ? R - dd : dd + 1;
            T ym[VW], yp[VW];
            vload_row<T, YA, VW>(pl + s_c - d * nx, d, ym);
            vload_row<T, YA, VW>(pl + s_c + d * nx, d, yp);
            const float2 cd = make_float2(A.c[d - 1], A.c[d - 1]);
            const int sm = (u + R - d) % Q, sp = (u + R + d) % Q;
#pragma unroll
            for (int h = 0; h < NP; ++h) {
              const int j = 2 * h;
              const float2 yy = __fadd2_rn(make_float2(ym[j], ym[j + 1]), make_float2(yp[j], yp[j + 1]));
              const float2 zz = __fadd2_rn(make_float2(zq[j][sm], zq[j + 1][sm]), make_float2(zq[j][sp], zq[j + 1][sp]));
              float2 xx;
              if constexpr (PAIRM) {
                const float* xw = h == 0 ? xa : xb;
                xx = __fadd2_rn(make_float2(xw[OFF + j - d], xw[OFF + j + 1 - d]),
                                make_float2(xw[OFF + j + d], xw[OFF + j + 1 + d]));
              } else {
                xx = __fadd2_rn(make_float2(xl(j, d), xl(j + 1, d)), make_float2(xr(j, d), xr(j + 1, d)));
              }
              const float2 t = __fadd2_rn(__fadd2_rn(yy, zz), xx);
              acc[h] = __ffma2_rn(cd, t, acc[h]);
            }
          }
#pragma unroll
          for (int h = 0; h < NP; ++h) {
            const int j = 2 * h;
            const float2 xc = make_float2(xs[OFF + j], xs[OFF + j + 1]);
            float2 a = acc[h];
            if constexpr (REV) a = __ffma2_rn(make_float2(c0, c0), xc, a);
            if constexpr (COMP) a = __ffma2_rn(make_float2(A.csr, A.csr), xc, a);
            if (has_pot) a = __ffma2_rn(make_float2(pov[j], pov[j + 1]), xc, a);
            float2 r = __ffma2_rn(make_float2(ca, ca), a, __fmul2_rn(make_float2(cb, cb), xc));
            if (Pc) r = __ffma2_rn(make_float2(cg, cg), make_float2(pvv[j], pvv[j + 1]), r);
            o[j] = r.x;
            o[j + 1] = r.y;
          }
        } else {
          T acc[VW];
#pragma unroll
          for (int j = 0; j < VW; ++j) acc[j] = REV ? T(0) : c0 * xs[OFF + j];
#pragma unroll
          for (int dd = 0; dd < R; ++dd) {
            const int d = REV ? R - dd : dd + 1;
            T ym[VW], yp[VW];
            vload_row<T, YA, VW>(pl + s_c - d * nx, d, ym);
            vload_row<T, YA, VW>(pl + s_c + d * nx, d, yp);
            const T cd = A.c[d - 1];
#pragma unroll
            for (int j = 0; j < VW; ++j) {
              const T t = ((ym[j] + yp[j]) + (zq[j][(u + R - d) % Q] + zq[j][(u + R + d) % Q])) +
                          (xl(j, d) + xr(j, d));
              acc[j] += cd * t;
            }
          }
#pragma unroll
          for (int j = 0; j < VW; ++j) {
            const T xc = xs[OFF + j];
            T a = acc[j];
            if constexpr (REV) a += c0 * xc;
            if constexpr (COMP) a += A.csr * xc;
            if (has_pot) a += pov[j] * xc;
            o[j] = ca * a + cb * xc;
            if (Pc) o[j] += cg * pvv[j];
          }
        }
        if (masked) {
          const double zm = z * A.h - A.cz;
#pragma unroll
          for (int j = 0; j < VW; ++j)
            if (mxy[j] + zm * zm > A.mask_r2) o[j] = T(0);
        }
        vstore<VW>(Yc + (long)z * nxy + q, o);
      }
      // every SYNC_EVERY planes (and after the last): the slots of all
      // planes <= z are free, so the ring is topped up to plane z + NBUF.
      // The queue front z + R stays covered while SYNC_EVERY <= NBUF - R.
      if ((z - z0) % SYNC_EVERY == SYNC_EVERY - 1 || z == z1 - 1) {
        __syncthreads();
        if (threadIdx.x == 0 && !fail)
          for (; issued < zlast && issued <= z + NBUF; ++issued) issue_x(issued);
      }
    }
  }
  if (fail) s_fail = 1;
  // Thread 0 issues every copy and waits for the planes in order; once it
  // has given up it issues no more, so the planes fail_plane .. issued-1 sit
  // in distinct slots.  Their copies are drained before the CTA exits.
  if (threadIdx.x == 0 && fail)
    for (int p = fail_plane; p < issued; ++p)
      mbar_wait(&bars[(p - z0) % NBUF], ((p - z0) / NBUF) & 1, PSC_DRAIN_WAIT);
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
  if (((uintptr_t)X | (uintptr_t)Y | (uintptr_t)P) % 16) return false;
  return true;
}

// Work table of one launch.  A CTA owns (column, slab, z range); the cost of a
// CTA is modelled as its planes plus a pipeline fill.  CTAs are dispatched
// about in order as resident slots free up, so the table puts whole-column
// (or half-column) items first and splits the last m (column, slab) pairs
// into smaller z chunks that fill the final wave.  The split is the one with
// the shortest simulated list-scheduling makespan over `slots` resident CTAs.
static void z_chunks(int nz, int c, std::vector<int2>& out) {
  const int zc = (nz + c - 1) / c;
  out.clear();
  for (int z = 0; z < nz; z += zc) out.push_back(make_int2(z, std::min(nz, z + zc)));
}

static double makespan(const std::vector<int>& cost, int slots) {
  std::priority_queue<double, std::vector<double>, std::greater<double>> q;
  for (int i = 0; i < slots; ++i) q.push(0.0);
  double end = 0.0;
  for (int c : cost) {
    const double t = q.top() + c;
    q.pop();
    q.push(t);
    end = std::max(end, t);
  }
  return end;
}

static std::vector<int4> stencil_schedule(int nslab, int nz, int k, int fill, int slots) {
  const long pairs = (long)nslab * k;
  const int cmax = std::max(1, nz / 8);  // chunks of at least 8 planes
  double best = 1e300;
  int bb = 1, bs = 1;
  long bm = 0;
  std::vector<int2> cb, cs;
  std::vector<int> cost;
  for (int b = 1; b <= std::min(2, cmax); ++b) {
    for (int sm = 1; sm <= 4; ++sm) {
      const int sc = std::min(cmax, b * sm);
      if (sm > 1 && sc == b) continue;
      z_chunks(nz, b, cb);
      z_chunks(nz, sc, cs);
      const long step = std::max(1L, pairs / 32);
      for (long m = 0; m <= pairs; m += step) {
        if (sc == b && m > 0) break;
        cost.clear();
        for (long p = 0; p < pairs - m; ++p)
          for (const int2& c : cb) cost.push_back(c.y - c.x + fill);
        for (long p = 0; p < m; ++p)
          for (const int2& c : cs) cost.push_back(c.y - c.x + fill);
        const double t = makespan(cost, slots);
        if (t < best - 1e-9) {
          best = t;
          bb = b;
          bs = sc;
          bm = m;
        }
      }
    }
  }
  z_chunks(nz, bb, cb);
  z_chunks(nz, bs, cs);
  std::vector<int4> out;
  for (long p = 0; p < pairs; ++p) {
    const int col = (int)(p / nslab), slab = (int)(p % nslab);
    for (const int2& c : (p < pairs - bm ? cb : cs)) out.push_back(make_int4(col, slab, c.x, c.y));
  }
  return out;
}

// Masked launches (sphere mode): per slab, the planes [zlo, zhi) that hold a
// point inside the sphere (one plane of margin each side) are computed, the
// rest only zero-filled.  Compute items are cut into chunks of at most lc
// planes and sorted longest first; the zero items (column stored as
// -1 - column) follow, at about a third of a plane's cost each.
static std::vector<int4> stencil_schedule_masked(const psc_ctx* ctx, int ts, int nslab, int k, int slots) {
  const int nx = ctx->nx, nxy = ctx->nx * ctx->ny, nz = ctx->nz;
  std::vector<int2> zr(nslab);
  long work = 0;
  for (int sl = 0; sl < nslab; ++sl) {
    double d2 = 1e300;
    for (int q = sl * ts; q < std::min(nxy, (sl + 1) * ts); ++q) {
      const double x = (q % nx) * ctx->h - ctx->mask_c[0], y = (q / nx) * ctx->h - ctx->mask_c[1];
      d2 = std::min(d2, x * x + y * y);
    }
    int lo = nz, hi = 0;
    if (d2 <= ctx->mask_r2) {
      const double half = std::sqrt(ctx->mask_r2 - d2);
      lo = std::max(0, (int)std::floor((ctx->mask_c[2] - half) / ctx->h) - 1);
      hi = std::min(nz, (int)std::ceil((ctx->mask_c[2] + half) / ctx->h) + 2);
    }
    zr[sl] = make_int2(lo, hi);
    if (hi > lo) work += hi - lo;
  }
  const int lc = std::max(8, (int)std::min<long>(nz, (work * (long)k + 2L * slots - 1) / (2L * slots)));
  std::vector<int4> comp, zero;
  for (int col = 0; col < k; ++col)
    for (int sl = 0; sl < nslab; ++sl) {
      const int lo = zr[sl].x, hi = zr[sl].y;
      if (hi > lo) {
        const int nch = (hi - lo + lc - 1) / lc;
        const int len = (hi - lo + nch - 1) / nch;
        for (int z = lo; z < hi; z += len) comp.push_back(make_int4(col, sl, z, std::min(hi, z + len)));
        if (lo > 0) zero.push_back(make_int4(-1 - col, sl, 0, lo));
        if (hi < nz) zero.push_back(make_int4(-1 - col, sl, hi, nz));
      } else {
        zero.push_back(make_int4(-1 - col, sl, 0, nz));
      }
    }
  std::stable_sort(comp.begin(), comp.end(), [](const int4& a, const int4& b) { return a.w - a.z > b.w - b.z; });
  comp.insert(comp.end(), zero.begin(), zero.end());
  return comp;
}

// Cached per context: the table of a (k, slab count, fill, mask) combination
// is built and uploaded once.
static const int4* stencil_sched(psc_ctx* ctx, int nslab, int k, int fill, int slots, bool masked, int ts, int* n,
                                 cudaStream_t st) {
  const long long key = ((long long)k << 32) | ((long long)nslab << 16) | ((long long)fill << 8) | (slots & 0x7f) |
                        (masked ? 0x80 : 0);
  for (auto& e : ctx->st_sched)
    if (e.key == key) {
      *n = e.n;
      return reinterpret_cast<const int4*>(e.dev);
    }
  psc_ctx::StencilSched e;
  e.key = key;
  std::vector<int4> tab = masked ? stencil_schedule_masked(ctx, ts, nslab, k, slots)
                                 : stencil_schedule(nslab, ctx->nz, k, fill, slots);
  e.n = (int)tab.size();
  e.host.resize(4 * tab.size());
  std::memcpy(e.host.data(), tab.data(), tab.size() * sizeof(int4));
  if (psc_dmalloc(&e.dev, tab.size() * sizeof(int4)) != cudaSuccess) return nullptr;
  ctx->st_sched.push_back(std::move(e));
  auto& b = ctx->st_sched.back();
  if (cudaMemcpyAsync(b.dev, b.host.data(), b.host.size() * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return nullptr;
  *n = b.n;
  return reinterpret_cast<const int4*>(b.dev);
}

template <typename T, int R, int VW, int MODE>
static int launch_tma_t(psc_ctx* ctx, int k, const T* X, long ldx, const T* P, long ldp, T* Y, long ldy,
                        const T* pot, const double* w, const double* coef, double a, double b, double g,
                        bool masked, cudaStream_t st) {
  const int nxy = ctx->nx * ctx->ny;
  constexpr int TS = slab_points<VW>();
  const int nslab = (nxy + TS - 1) / TS;
  // each CTA pays a pipeline fill of about R + D planes; two CTAs per SM
  // are resident (registers and shared memory)
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int slots = PSC_STENCIL_CTAS_PER_SM * sms;
  const int fill = R + prefetch_depth<T>() + 2;
  int nwork = 0;
  masked = masked && ctx->mask_r2 > 0.0;
  const int4* sched = stencil_sched(ctx, nslab, k, fill, slots, masked, TS, &nwork, st);
  PSC_REQUIRE(ctx, sched != nullptr, "stencil: work table allocation failed");
  constexpr int NBUF = R + 1 + prefetch_depth<T>();
  constexpr size_t Q16 = 16 / sizeof(T);
  const size_t win = (TS + 2 * (size_t)R * ctx->nx + VW + Q16 - 1) / Q16 * Q16;   // window + zero pad, 16-byte slots
  const size_t smem = (NBUF * win + (size_t)PP_SLOTS * 2 * TS) * sizeof(T) + NBUF * sizeof(uint64_t);
  if (smem > 220 * 1024) return -1;  // window too wide: the register-queue kernel takes it
  auto kern = (ctx->nx % VW == 0) ? k_stencil_tma<T, R, VW, VW, MODE>
              : (ctx->nx % 2 == 0) ? k_stencil_tma<T, R, (VW >= 2 ? 2 : 1), VW, MODE>
                                   : k_stencil_tma<T, R, 1, VW, MODE>;
  PSC_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  TmaArgs<T> A;
  A.X = X; A.ldx = ldx; A.P = P; A.ldp = ldp; A.Y = Y; A.ldy = ldy; A.pot = pot;
  A.nx = ctx->nx; A.ny = ctx->ny; A.nz = ctx->nz; A.sched = sched;
  A.c0 = (T)w[0];
  // the sum rule c0 + 6 sum_d c_d = 0 holds for the FP64 weights; in the
  // stored type it is off by the weights' rounding errors, which the
  // correction term removes (FP32 only, MODE bit 1)
  double rs = (double)A.c0 - w[0];
  for (int i = 0; i < 4; ++i) {
    A.c[i] = (T)w[1 + i];
    rs += 6.0 * ((double)A.c[i] - w[1 + i]);
  }
  A.csr = (T)(-rs);
  A.coef = coef; A.a = a; A.b = b; A.g = g; A.status = ctx->dev_status;
  A.wait_limit = ctx->wait_limit;
  A.mask_r2 = masked ? ctx->mask_r2 : 0.0;
  A.h = ctx->h;
  A.cx = ctx->mask_c[0]; A.cy = ctx->mask_c[1]; A.cz = ctx->mask_c[2];
  kern<<<nwork, TNT, smem, st>>>(A);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

// Returns -1 if the TMA path does not apply (caller uses the register kernel).
template <typename T>
int psc_stencil_tma(psc_ctx* ctx, int k, const T* X, long ldx, const T* P, long ldp, T* Y, long ldy, const T* pot,
                    const double* w, const double* coef, double a, double b, double g, bool masked,
                    cudaStream_t st) {
  if (!tma_ok<T>(ctx, X, ldx, P, ldp, Y, ldy)) return -1;
  // FP32 takes 4-point runs with the arithmetic on packed pairs (measured
  // fastest, also where nx is only 2-aligned and the x terms need per-point
  // edge masks: 818 us per step at 90^3, k = 307, against 995-1055 us for
  // 2-point runs and 894 us for scalar arithmetic); impl 2 / 3 ask for
  // 2-point runs when nx is even but not a multiple of 4, impl 3 / 4 for
  // scalar arithmetic
  const int impl = ctx->stencil_impl;
  const bool narrow = sizeof(T) == 4 && ctx->nx % 4 != 0 && ctx->nx % 2 == 0 && (impl == 2 || impl == 3);
  // the correction term in the kernel: weights mode 1, or mode 2 when this
  // call's potential is not the FP32 potential that carries it
  const bool comp = ctx->stencil_comp == 1 ||
                    (ctx->stencil_comp == 2 && (const void*)pot != (const void*)ctx->pot32);
  const int mode = (impl == 0 || impl == 2 ? 1 : 0) | (comp ? 2 : 0);
#define PSC_TMA_ARGS ctx, k, X, ldx, P, ldp, Y, ldy, pot, w, coef, a, b, g, masked, st
#define PSC_TMA_MODES(VWW)                                                                                    \
  switch (mode) {                                                                                             \
    case 0: return launch_tma_t<T, RR, VWW, 0>(PSC_TMA_ARGS);                                                 \
    case 1: return launch_tma_t<T, RR, VWW, 1>(PSC_TMA_ARGS);                                                 \
    case 2: return launch_tma_t<T, RR, VWW, 2>(PSC_TMA_ARGS);                                                 \
    default: return launch_tma_t<T, RR, VWW, 3>(PSC_TMA_ARGS);                                                \
  }
#define PSC_TMA_R(RRV)                                                                                        \
  case RRV: {                                                                                                 \
    constexpr int RR = RRV;                                                                                   \
    if constexpr (sizeof(T) == 8)                                                                             \
      return launch_tma_t<T, RR, 2, 0>(PSC_TMA_ARGS);                                                         \
    else if (narrow) {                                                                                        \
      PSC_TMA_MODES(2)                                                                                        \
    } else {                                                                                                  \
      PSC_TMA_MODES(4)                                                                                        \
    }                                                                                                         \
  }
  switch (ctx->radius) {
    PSC_TMA_R(1)
    PSC_TMA_R(2)
    PSC_TMA_R(3)
    PSC_TMA_R(4)
  }
#undef PSC_TMA_R
#undef PSC_TMA_MODES
#undef PSC_TMA_ARGS
  return -1;
}

template int psc_stencil_tma<double>(psc_ctx*, int, const double*, long, const double*, long, double*, long,
                                     const double*, const double*, const double*, double, double, double, bool,
                                     cudaStream_t);
template int psc_stencil_tma<float>(psc_ctx*, int, const float*, long, const float*, long, float*, long,
                                    const float*, const double*, const double*, double, double, double, bool,
                                    cudaStream_t);
