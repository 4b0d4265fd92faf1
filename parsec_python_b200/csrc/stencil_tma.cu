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
// Every mbarrier wait is bounded: on timeout the CTA records the failure in
// status[3] and carries on without waiting (results are then garbage but the
// GPU is never hung).  Every bulk copy issued is waited for before the CTA
// exits.
#include "psc_internal.cuh"
#include "../../include/psc.h"

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

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
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

// 16-byte vectors: two FP64 or four FP32 points per thread
template <typename T>
struct VecOf;
template <>
struct VecOf<double> {
  using type = double2;
  static constexpr int W = 2;
};
template <>
struct VecOf<float> {
  using type = float4;
  static constexpr int W = 4;
};

template <typename T>
__device__ __forceinline__ void vload(const T* p, T* out) {
  using V = typename VecOf<T>::type;
  const V v = *reinterpret_cast<const V*>(p);
  const T* e = reinterpret_cast<const T*>(&v);
#pragma unroll
  for (int j = 0; j < VecOf<T>::W; ++j) out[j] = e[j];
}

template <typename T>
__device__ __forceinline__ void vstore(T* p, const T* in) {
  using V = typename VecOf<T>::type;
  V v;
  T* e = reinterpret_cast<T*>(&v);
#pragma unroll
  for (int j = 0; j < VecOf<T>::W; ++j) e[j] = in[j];
  *reinterpret_cast<V*>(p) = v;
}

// load VW consecutive values from an address aligned to A elements (A | VW)
template <typename T, int A>
__device__ __forceinline__ void vload_a(const T* p, T* out) {
  constexpr int VW = VecOf<T>::W;
  if constexpr (A == VW) {
    vload(p, out);
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

template <typename T>
__host__ __device__ constexpr int slab_points() {
  return VecOf<T>::W * TNT;
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
  const double* coef;
  double a, b, g;
  int* status;
};

}  // namespace

// YA: alignment (in elements) of the y-neighbour rows, the largest of VW, 2, 1
// that divides nx; their loads are split to match.
template <typename T, int R, int YA>
__global__ void __launch_bounds__(TNT)
k_stencil_tma(TmaArgs<T> A) {
  constexpr int VW = VecOf<T>::W;          // points per thread
  constexpr int TS = slab_points<T>();     // points per slab
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
  const int WS = WIN + VW;  // slot stride: the window and one zero vector
  T* ring = reinterpret_cast<T*>(smem_raw);                                   // [NBUF][WS]
  T* pring = ring + (size_t)NBUF * WS;                                        // [NS][2][TS]: Prev, pot
  uint64_t* bars = reinterpret_cast<uint64_t*>(pring + (size_t)NS * 2 * TS);  // [NBUF]
  __shared__ int s_fail;

  const int4 work = A.sched[blockIdx.x];
  const int slab0 = work.y * TS;
  const int z0 = work.z;
  const int z1 = work.w;
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
      if (Pc) cp_async16(d, Pc + (long)z * nxy + q);
      if (has_pot) cp_async16(d + TS, A.pot + (long)z * nxy + q);
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
      vload(Xc + (long)zz * nxy + q, v);
#pragma unroll
      for (int j = 0; j < VW; ++j) zq[j][i] = v[j];
    }
  }
  bool fail = false;
#pragma unroll
  for (int i = 0; i < R; ++i) {
    const int p = z0 + i;
    if (p < nz) {
      const int s = (p - z0) % NBUF;
      if (!fail && !mbar_wait(&bars[s], ((p - z0) / NBUF) & 1)) fail = true;
      if (own) {
        T v[VW];
        vload(ring + (size_t)s * WS + s_c, v);
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
          if (!fail && !mbar_wait(&bars[s], ((pf - z0) / NBUF) & 1)) fail = true;
          if (own) vload(ring + (size_t)s * WS + s_c, f);
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
          if (Pc) vload(pp, pvv);
          if (has_pot) vload(pp + TS, pov);
        }
      }
      const T* pl = ring + (size_t)((z - z0) % NBUF) * WS;
      if (EXACT && own) {
        T xs[NPV * VW];
#pragma unroll
        for (int v = 0; v < NPV; ++v) {
          if (v == HV) {
#pragma unroll
            for (int j = 0; j < VW; ++j) xs[v * VW + j] = zq[j][(u + R) % Q];
          } else {
            vload(pl + xo[v], xs + v * VW);
          }
        }
        const T* pc = pl + s_c;
        T acc[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) acc[j] = c0 * xs[OFF + j];
#pragma unroll
        for (int d = 1; d <= R; ++d) {
          T ym[VW], yp[VW];
          vload(pc - d * nx, ym);
          vload(pc + d * nx, yp);
          const T cd = A.c[d - 1];
#pragma unroll
          for (int j = 0; j < VW; ++j) {
            const T t = ((ym[j] + yp[j]) + (zq[j][(u + R - d) % Q] + zq[j][(u + R + d) % Q])) +
                        (xs[OFF + j - d] + xs[OFF + j + d]);
            acc[j] += cd * t;
          }
        }
        T o[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) {
          const T xc = xs[OFF + j];
          T a = acc[j];
          if (has_pot) a += pov[j] * xc;
          o[j] = ca * a + cb * xc;
          if (Pc) o[j] += cg * pvv[j];
        }
        vstore(Yc + (long)z * nxy + q, o);
      } else if (own) {
        // x neighbours: the aligned vectors around the run; the run itself is the queue's centre
        T xs[NPV * VW];
#pragma unroll
        for (int v = 0; v < NPV; ++v) {
          if (v == HV) {
#pragma unroll
            for (int j = 0; j < VW; ++j) xs[v * VW + j] = zq[j][(u + R) % Q];
          } else {
            vload(pl + s_c - OFF + v * VW, xs + v * VW);
          }
        }
        // two partial sums per point: y + z terms, x terms
        T acc[VW], ax[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) {
          acc[j] = c0 * xs[OFF + j];
          ax[j] = T(0);
        }
#pragma unroll
        for (int d = 1; d <= R; ++d) {
          // rows outside the plane are zero in the window, so y needs no test
          T ym[VW], yp[VW];
          vload_a<T, YA>(pl + s_c - d * nx, ym);
          vload_a<T, YA>(pl + s_c + d * nx, yp);
          const T cd = A.c[d - 1];
#pragma unroll
          for (int j = 0; j < VW; ++j) {
            const T t = (ym[j] + yp[j]) + (zq[j][(u + R - d) % Q] + zq[j][(u + R + d) % Q]);
            acc[j] += cd * t;
            const T xsum = (d <= el[j] ? xs[OFF + j - d] : T(0)) + (d <= er[j] ? xs[OFF + j + d] : T(0));
            ax[j] += cd * xsum;
          }
        }
        T o[VW];
#pragma unroll
        for (int j = 0; j < VW; ++j) {
          const T xc = xs[OFF + j];
          T a = acc[j] + ax[j];
          if (has_pot) a += pov[j] * xc;
          o[j] = ca * a + cb * xc;
          if (Pc) o[j] += cg * pvv[j];
        }
        vstore(Yc + (long)z * nxy + q, o);
      }
      // every SYNC_EVERY planes (and after the last): the slots of all
      // planes <= z are free, so the ring is topped up to plane z + NBUF.
      // The queue front z + R stays covered while SYNC_EVERY <= NBUF - R.
      if ((z - z0) % SYNC_EVERY == SYNC_EVERY - 1 || z == z1 - 1) {
        __syncthreads();
        if (threadIdx.x == 0)
          for (; issued < zlast && issued <= z + NBUF; ++issued) issue_x(issued);
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

// Cached per context: the table of a (k, slab count, fill) combination is
// built and uploaded once.
static const int4* stencil_sched(psc_ctx* ctx, int nslab, int k, int fill, int slots, int* n, cudaStream_t st) {
  const long long key = ((long long)k << 32) | ((long long)nslab << 16) | ((long long)fill << 8) | (slots & 0xff);
  for (auto& e : ctx->st_sched)
    if (e.key == key) {
      *n = e.n;
      return reinterpret_cast<const int4*>(e.dev);
    }
  psc_ctx::StencilSched e;
  e.key = key;
  std::vector<int4> tab = stencil_schedule(nslab, ctx->nz, k, fill, slots);
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

template <typename T, int R>
static int launch_tma_t(psc_ctx* ctx, int k, const T* X, long ldx, const T* P, long ldp, T* Y, long ldy,
                        const T* pot, const double* w, const double* coef, double a, double b, double g,
                        cudaStream_t st) {
  const int nxy = ctx->nx * ctx->ny;
  constexpr int TS = slab_points<T>();
  const int nslab = (nxy + TS - 1) / TS;
  // each CTA pays a pipeline fill of about R + D planes; two CTAs per SM
  // are resident (registers and shared memory)
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int slots = PSC_STENCIL_CTAS_PER_SM * sms;
  const int fill = R + prefetch_depth<T>() + 2;
  int nwork = 0;
  const int4* sched = stencil_sched(ctx, nslab, k, fill, slots, &nwork, st);
  PSC_REQUIRE(ctx, sched != nullptr, "stencil: work table allocation failed");
  constexpr int NBUF = R + 1 + prefetch_depth<T>();
  const size_t win = TS + 2 * (size_t)R * ctx->nx + VecOf<T>::W;   // window + zero pad vector
  const size_t smem = (NBUF * win + (size_t)PP_SLOTS * 2 * TS) * sizeof(T) + NBUF * sizeof(uint64_t);
  if (smem > 220 * 1024) return -1;  // window too wide: the register-queue kernel takes it
  constexpr int VW = VecOf<T>::W;
  auto kern = (ctx->nx % VW == 0) ? k_stencil_tma<T, R, VW>
              : (ctx->nx % 2 == 0) ? k_stencil_tma<T, R, (VW >= 2 ? 2 : 1)>
                                   : k_stencil_tma<T, R, 1>;
  PSC_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  TmaArgs<T> A;
  A.X = X; A.ldx = ldx; A.P = P; A.ldp = ldp; A.Y = Y; A.ldy = ldy; A.pot = pot;
  A.nx = ctx->nx; A.ny = ctx->ny; A.nz = ctx->nz; A.sched = sched;
  A.c0 = (T)w[0];
  for (int i = 0; i < 4; ++i) A.c[i] = (T)w[1 + i];
  A.coef = coef; A.a = a; A.b = b; A.g = g; A.status = ctx->dev_status;
  kern<<<nwork, TNT, smem, st>>>(A);
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
