// Hartree solve: conjugate gradients on A = -Lap_h (Eigensolvers/pcg.py:7-85),
// warm started, stop when r.r <= tol^2 * r0.r0 or after maxit iterations.
//
// Two launches per iteration, all scalars on the device:
//   A  every CTA re-reduces the r.r partials of the previous iteration (fixed
//      order, so all CTAs agree bit for bit), takes the stop decision,
//      beta = ro1/ro, and applies the stencil to the new direction
//      p = r + beta q computed at every load (q = previous p; q = r in the
//      second iteration, because in the reference the first direction aliases
//      the residual array and its first update is p = (1 + beta) r; p = r in
//      the first).  It writes p and Ap for its own points and a partial of
//      p.Ap.  The two p buffers alternate between iterations.
//   B  alpha = ro / pAp (again reduced by every CTA), x += alpha p,
//      r -= alpha Ap, partial of r.r.
// Scalars that a kernel reads are only ever written by the other kernel (or
// by init), so no CTA reads a value that another CTA of the same launch is
// writing.  Eight iterations are captured once per context as a CUDA graph
// and replayed; once the stop decision is taken both kernels return at once.
// The host reads the "active" flag between replays.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>

// scalar slots (ctx->scalars)
#define CG_IT_A 64     // iteration kernel A performs next (written by B / init)
#define CG_IT_B 65     // iteration kernel B performs next (written by A)
#define CG_TOL1 66
#define CG_ACTIVE 67
#define CG_ITS 68      // completed iterations (written by B)
#define CG_MAXIT 69
#define CG_RO_SLOTS 512  // ro per iteration: ctx->cg_ro[it] = r.r before iteration it

constexpr int CG_CHUNK = 8;   // iterations per graph replay (even: the p buffers alternate)
constexpr int CG_NT = 256;
constexpr int CG_ZCHUNK = 8;

__global__ void k_cg_init(double* sc, double* ro_arr, const double* rr, double tol, int maxit) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const double ro1 = rr[0];
    ro_arr[1] = ro1;
    sc[CG_TOL1] = tol * tol * ro1;
    sc[CG_ITS] = 0.0;
    sc[CG_MAXIT] = (double)maxit;
    sc[CG_IT_A] = 1.0;
    sc[CG_IT_B] = 1.0;
    sc[CG_ACTIVE] = (0 < maxit && ro1 > tol * tol * ro1) ? 1.0 : 0.0;
  }
}

__device__ __forceinline__ double cg_reduce(const double* part, int np, double* sh, double* bc) {
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += CG_NT) s += part[i];
  s = psc_block_sum<double, CG_NT>(s, sh);
  if (threadIdx.x == 0) *bc = s;
  __syncthreads();
  return *bc;
}

// Kernel A: direction update fused into the Laplacian stencil (z-marching
// CTA over a slab of 256 flat xy points, register z queue, shared-memory plane).
template <int R>
__global__ void __launch_bounds__(CG_NT)
k_cg_dir_stencil(const double* __restrict__ r, const double* __restrict__ pold, double* __restrict__ pnew,
                 double* __restrict__ ap, int nx, int ny, int nz, double c0, double4 cw, double* sc,
                 double* ro_arr, const double* __restrict__ part2, int np2, double* __restrict__ part1) {
  extern __shared__ double plane[];
  __shared__ double sh[CG_NT / 32];
  __shared__ double bc;
  __shared__ double s_act, s_it;
  // one thread reads the flags (CTA 0 may clear "active" during this launch),
  // so every thread of a CTA takes the same path
  if (threadIdx.x == 0) { s_act = sc[CG_ACTIVE]; s_it = sc[CG_IT_A]; }
  __syncthreads();
  if (s_act == 0.0) return;
  const int it = (int)s_it;
  bool stop = it > (int)sc[CG_MAXIT];
  double beta = 0.0;
  bool alias = true;
  if (!stop && it >= 2) {
    const double ro1 = cg_reduce(part2, np2, sh, &bc);
    if (!(ro1 > sc[CG_TOL1])) {
      stop = true;
    } else {
      beta = ro1 / ro_arr[it - 1];
      alias = it == 2;
      if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) ro_arr[it] = ro1;
    }
  }
  if (stop) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) sc[CG_ACTIVE] = 0.0;
    return;
  }
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) sc[CG_IT_B] = (double)it;
  const double* q = alias ? r : pold;
  const double cd[4] = {cw.x, cw.y, cw.z, cw.w};

  const int nxy = nx * ny;
  const int halo = R * nx;
  const int S = CG_NT;
  const int win = S + 2 * halo;
  const int slab0 = blockIdx.x * S;
  const int seff = min(S, nxy - slab0);
  const int z0 = blockIdx.y * CG_ZCHUNK;
  const int z1 = min(nz, z0 + CG_ZCHUNK);
  const int loc = threadIdx.x;
  const bool own = loc < seff;
  const int qp = slab0 + loc;
  const int xi = own ? qp % nx : 0;
  const int yi = own ? qp / nx : 0;

  double zq[2 * R + 1];
#pragma unroll
  for (int i = 0; i < 2 * R; ++i) {
    const int zz = z0 - R + i;
    double v = 0.0;
    if (own && zz >= 0 && zz < nz) {
      const long g = (long)zz * nxy + qp;
      v = r[g] + beta * q[g];
    }
    zq[i] = v;
  }
  double dacc = 0.0;
  int buf = 0;
  const int hcount = win - seff;
  for (int z = z0; z < z1; ++z) {
    double* pl = plane + buf * win;
    const long zoff = (long)z * nxy;
    {
      const int zz = z + R;
      double v = 0.0;
      if (own && zz < nz) {
        const long g = (long)zz * nxy + qp;
        v = r[g] + beta * q[g];
      }
      zq[2 * R] = v;
      if (own) pl[halo + loc] = zq[R];
    }
    for (int j = threadIdx.x; j < hcount; j += CG_NT) {
      const int pos = j < halo ? j : j + seff;
      const int fq = slab0 - halo + pos;
      double v = 0.0;
      if (fq >= 0 && fq < nxy) v = r[zoff + fq] + beta * q[zoff + fq];
      pl[pos] = v;
    }
    __syncthreads();
    if (own) {
      const int s = halo + loc;
      const double xc = zq[R];
      double acc = c0 * xc;
#pragma unroll
      for (int d = 1; d <= R; ++d) {
        double sx = 0.0, sy = 0.0;
        if (xi - d >= 0) sx += pl[s - d];
        if (xi + d < nx) sx += pl[s + d];
        if (yi - d >= 0) sy += pl[s - d * nx];
        if (yi + d < ny) sy += pl[s + d * nx];
        acc += cd[d - 1] * (sx + sy + (zq[R - d] + zq[R + d]));
      }
      pnew[zoff + qp] = xc;
      ap[zoff + qp] = acc;
      dacc += acc * xc;
    }
#pragma unroll
    for (int i = 0; i < 2 * R; ++i) zq[i] = zq[i + 1];
    buf ^= 1;
  }
  dacc = psc_block_sum<double, CG_NT>(dacc, sh);
  if (threadIdx.x == 0) part1[(long)blockIdx.y * gridDim.x + blockIdx.x] = dacc;
}

// Kernel B: alpha, x and r updates, partial of r.r.
__global__ void __launch_bounds__(CG_NT)
k_cg_update(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
            const double* __restrict__ ap, long n, double* sc, const double* ro_arr,
            const double* __restrict__ part1, int np1, double* __restrict__ part2) {
  __shared__ double sh[CG_NT / 32];
  __shared__ double bc;
  __shared__ double s_act, s_it;
  if (threadIdx.x == 0) { s_act = sc[CG_ACTIVE]; s_it = sc[CG_IT_B]; }
  __syncthreads();
  if (s_act == 0.0) return;
  const int it = (int)s_it;
  const double pap = cg_reduce(part1, np1, sh, &bc);
  const double alp = ro_arr[it] / pap;
  double rr = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    x[i] += alp * p[i];
    const double ri = r[i] - alp * ap[i];
    r[i] = ri;
    rr += ri * ri;
  }
  rr = psc_block_sum<double, CG_NT>(rr, sh);
  if (threadIdx.x == 0) {
    part2[blockIdx.x] = rr;
    if (blockIdx.x == 0) {
      sc[CG_IT_A] = (double)(it + 1);
      sc[CG_ITS] = (double)it;
    }
  }
}

struct CgPlan {
  dim3 grid;
  size_t smem;
};

static CgPlan cg_plan(const psc_ctx* ctx) {
  CgPlan p;
  const int nxy = ctx->nx * ctx->ny;
  p.grid = dim3((nxy + CG_NT - 1) / CG_NT, (ctx->nz + CG_ZCHUNK - 1) / CG_ZCHUNK);
  p.smem = 2 * (size_t)(CG_NT + 2 * ctx->radius * ctx->nx) * sizeof(double);
  return p;
}

static int cg_iterations(psc_ctx* ctx, int count, cudaStream_t st) {
  const long n = ctx->n;
  const CgPlan pl = cg_plan(ctx);
  const int np1 = (int)(pl.grid.x * pl.grid.y);
  double* part1 = ctx->cg_part;
  double* part2 = ctx->cg_part + ctx->cg_part_cap;
  double* pbuf[2] = {ctx->cg_p, ctx->cg_p2};
  const double4 cw = make_double4(ctx->lap_c[0], ctx->lap_c[1], ctx->lap_c[2], ctx->lap_c[3]);
  for (int i = 0; i < count; ++i) {
    // chunks start at odd iterations: odd iterations (even i) write pbuf[1] and
    // read pbuf[0], even iterations the other way round
    const double* pold = pbuf[i & 1];
    double* pnew = pbuf[(i & 1) ^ 1];
#define PSC_CG_A(RR)                                                                                     \
  if (ctx->radius == RR) {                                                                               \
    if (pl.smem > 40 * 1024)                                                                             \
      PSC_CUDA(ctx, cudaFuncSetAttribute(k_cg_dir_stencil<RR>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                         (int)pl.smem));                                                 \
    k_cg_dir_stencil<RR><<<pl.grid, CG_NT, pl.smem, st>>>(ctx->cg_r, pold, pnew, ctx->cg_ap, ctx->nx, ctx->ny, \
                                                          ctx->nz, ctx->lap_c0, cw, ctx->scalars, ctx->cg_ro,  \
                                                          part2, PSC_RED_BLOCKS, part1);                 \
  }
    PSC_CG_A(1) else PSC_CG_A(2) else PSC_CG_A(3) else PSC_CG_A(4)
#undef PSC_CG_A
    PSC_LAUNCH_CHECK(ctx);
    k_cg_update<<<PSC_RED_BLOCKS, CG_NT, 0, st>>>(ctx->cg_x, ctx->cg_r, pnew, ctx->cg_ap, n, ctx->scalars,
                                                  ctx->cg_ro, part1, np1, part2);
    PSC_LAUNCH_CHECK(ctx);
  }
  return 0;
}

static int cg_graph(psc_ctx* ctx) {
  if (ctx->cg_exec) return 0;
  if (!ctx->cap_stream) PSC_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
  PSC_CUDA(ctx, cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal));
  const int rc = cg_iterations(ctx, CG_CHUNK, ctx->cap_stream);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(ctx->cap_stream, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  PSC_CUDA(ctx, e);
  const cudaError_t e2 = cudaGraphInstantiate(&ctx->cg_exec, g, 0);
  cudaGraphDestroy(g);
  PSC_CUDA(ctx, e2);
  return 0;
}

int psc_pcg_persistent(psc_ctx* ctx, const double* rhs, double* x, int maxit, double tol, int* its_out,
                       cudaStream_t st);

extern "C" int psc_pcg_poisson(psc_ctx* ctx, const double* rhs, double* x, int maxit, double tol, int* its_out,
                               void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, maxit >= 0 && maxit < CG_RO_SLOTS - 2, "pcg: maxit out of range (0..509)");
  cudaStream_t st = (cudaStream_t)stream;
  // one cooperative launch with the vectors resident in shared memory, when they fit
  {
    const int prc = psc_pcg_persistent(ctx, rhs, x, maxit, tol, its_out, st);
    if (prc >= 0) return prc;
  }
  const long n = ctx->n;
  const CgPlan pl = cg_plan(ctx);
  const int need = std::max((int)(pl.grid.x * pl.grid.y), PSC_RED_BLOCKS);
  if (ctx->cg_part_cap < need) {
    psc_dfree(ctx->cg_part);
    ctx->cg_part = nullptr;
    PSC_CUDA(ctx, psc_dmalloc(&ctx->cg_part, 2 * (size_t)need * sizeof(double)));
    ctx->cg_part_cap = need;
  }
  if (!ctx->cg_x) PSC_CUDA(ctx, psc_dmalloc(&ctx->cg_x, n * sizeof(double)));
  if (!ctx->cg_p2) PSC_CUDA(ctx, psc_dmalloc(&ctx->cg_p2, n * sizeof(double)));
  if (!ctx->cg_ro) PSC_CUDA(ctx, psc_dmalloc(&ctx->cg_ro, CG_RO_SLOTS * sizeof(double)));
  double* sc = ctx->scalars;
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->cg_x, x, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  // r = rhs - A x
  int rc = psc_laplacian_fused(ctx, ctx->cg_x, rhs, ctx->cg_r, -1.0, 0.0, 1.0, nullptr, nullptr, st);
  if (rc) return rc;
  const double* rr_a[1] = {ctx->cg_r};
  rc = psc_dots(ctx, 1, rr_a, rr_a, n, sc + 70, st);
  if (rc) return rc;
  k_cg_init<<<1, 32, 0, st>>>(sc, ctx->cg_ro, sc + 70, tol, maxit);
  PSC_LAUNCH_CHECK(ctx);
  const bool use_graph = ctx->use_graphs;
  if (use_graph) {
    rc = cg_graph(ctx);
    if (rc) return rc;
  }
  for (int done = 0; done < maxit; done += CG_CHUNK) {
    if (use_graph) {
      PSC_CUDA(ctx, cudaGraphLaunch(ctx->cg_exec, st));
      // the graph's kernels are counted as launches too
      for (int i = 0; i < 2 * CG_CHUNK; ++i) psc_note_launch();
    } else {
      rc = cg_iterations(ctx, CG_CHUNK, st);
      if (rc) return rc;
    }
    PSC_CUDA(ctx, cudaMemcpyAsync(ctx->host_scalars + CG_ACTIVE, sc + CG_ACTIVE, 2 * sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    PSC_CUDA(ctx, cudaStreamSynchronize(st));
    if (ctx->host_scalars[CG_ACTIVE] == 0.0) break;
  }
  PSC_CUDA(ctx, cudaMemcpyAsync(x, ctx->cg_x, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (its_out) *its_out = (int)ctx->host_scalars[CG_ITS];
  return 0;
}

// mode 2 (default): persistent cooperative kernel when the CG vectors fit in
// shared memory, else graph replay; 1: graph replay of the two CG kernels;
// 0: the two CG kernels launched from the host.
extern "C" int psc_set_use_graphs(psc_ctx* ctx, int mode) {
  if (!ctx) return 2;
  ctx->use_graphs = mode >= 1 ? 1 : 0;
  ctx->cg_persistent = mode >= 2 ? 1 : 0;
  return 0;
}
