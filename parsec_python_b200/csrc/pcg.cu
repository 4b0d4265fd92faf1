// Hartree solve: conjugate gradients on A = -Lap_h (Eigensolvers/pcg.py:7-85),
// warm started, stop when r.r <= tol^2 * r0.r0 or after maxit iterations.
//
// Per iteration three launches, all scalars on the device:
//   1. Ap = A p with a per-CTA partial of p.Ap fused into the stencil;
//   2. every CTA re-reduces the partials in the same fixed order (so all CTAs
//      agree bit for bit), alpha = ro/pAp, x += alpha p, r -= alpha Ap, and a
//      per-CTA partial of r.r; CTA 0 advances the iteration counter;
//   3. every CTA re-reduces r.r, beta = ro1/ro, p = r + beta p.  In the
//      reference the first direction aliases the residual array, so its first
//      update is p = (1 + beta) r; that is reproduced here.
// The kernels take no per-iteration arguments (counter and scalars live on
// the device), so eight iterations are captured once per context as a CUDA
// graph on internal buffers and replayed; after convergence the kernels return
// at once.  The host reads the "active" flag between replays.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>

// scalar slots (ctx->scalars)
#define CG_RO 64       // r.r of the current direction
#define CG_RO_PREV 65  // r.r before the latest update (written by every CTA of step 2)
#define CG_TOL1 66
#define CG_ACTIVE 67
#define CG_ITS 68
#define CG_MAXIT 69

constexpr int CG_CHUNK = 8;

__global__ void k_cg_init(double* sc, const double* rr, double tol, int maxit) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const double ro1 = rr[0];
    sc[CG_RO] = ro1;
    sc[CG_RO_PREV] = ro1;
    sc[CG_TOL1] = tol * tol * ro1;
    sc[CG_ITS] = 0.0;
    sc[CG_MAXIT] = (double)maxit;
    sc[CG_ACTIVE] = (0 < maxit && ro1 > tol * tol * ro1) ? 1.0 : 0.0;
  }
}

template <int NT>
__device__ __forceinline__ double cg_sum_partials(const double* part, int np, double* sh) {
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += NT) s += part[i];
  s = psc_block_sum<double, NT>(s, sh);
  __shared__ double bc;
  if (threadIdx.x == 0) bc = s;
  __syncthreads();
  return bc;
}

__global__ void __launch_bounds__(256)
k_cg_update(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
            const double* __restrict__ ap, long n, double* sc, const double* __restrict__ part1, int np1,
            double* __restrict__ part2) {
  if (sc[CG_ACTIVE] == 0.0) return;
  __shared__ double sh[8];
  const double pap = cg_sum_partials<256>(part1, np1, sh);
  const double ro = sc[CG_RO];
  const double alp = ro / pap;
  double rr = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    x[i] += alp * p[i];
    const double ri = r[i] - alp * ap[i];
    r[i] = ri;
    rr += ri * ri;
  }
  rr = psc_block_sum<double, 256>(rr, sh);
  if (threadIdx.x == 0) {
    part2[blockIdx.x] = rr;
    sc[CG_RO_PREV] = ro;  // same value from every CTA
    if (blockIdx.x == 0) sc[CG_ITS] += 1.0;
  }
}

__global__ void __launch_bounds__(256)
k_cg_direction(double* __restrict__ p, const double* __restrict__ r, long n, double* sc,
               const double* __restrict__ part2, int np2) {
  if (sc[CG_ACTIVE] == 0.0) return;
  __shared__ double sh[8];
  const double ro1 = cg_sum_partials<256>(part2, np2, sh);
  const double ro = sc[CG_RO_PREV];
  const double bet = ro1 / ro;
  const double it = sc[CG_ITS];
  const bool first = it == 1.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double ri = r[i];
    p[i] = first ? ri + bet * ri : ri + bet * p[i];
  }
  // CTAs that start after CTA 0 cleared the flag skip the update of p, which
  // is then no longer used.
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc[CG_RO] = ro1;
    sc[CG_ACTIVE] = (it < sc[CG_MAXIT] && ro1 > sc[CG_TOL1]) ? 1.0 : 0.0;
  }
}

static int cg_iterations(psc_ctx* ctx, int count, cudaStream_t st) {
  const long n = ctx->n;
  double* part1 = ctx->cg_part;
  double* part2 = ctx->cg_part + ctx->cg_part_cap;
  for (int i = 0; i < count; ++i) {
    int nb = 0;
    int rc = psc_laplacian_fused(ctx, ctx->cg_p, nullptr, ctx->cg_ap, 1.0, 0.0, 0.0, part1, &nb, st);
    if (rc) return rc;
    k_cg_update<<<PSC_RED_BLOCKS, 256, 0, st>>>(ctx->cg_x, ctx->cg_r, ctx->cg_p, ctx->cg_ap, n, ctx->scalars, part1,
                                                nb, part2);
    PSC_LAUNCH_CHECK(ctx);
    k_cg_direction<<<PSC_RED_BLOCKS, 256, 0, st>>>(ctx->cg_p, ctx->cg_r, n, ctx->scalars, part2, PSC_RED_BLOCKS);
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

extern "C" int psc_pcg_poisson(psc_ctx* ctx, const double* rhs, double* x, int maxit, double tol, int* its_out,
                               void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, maxit >= 0, "pcg: maxit < 0");
  cudaStream_t st = (cudaStream_t)stream;
  const long n = ctx->n;
  const int nb1 = psc_stencil_blocks(ctx, 1);
  const int need = std::max(nb1, PSC_RED_BLOCKS);
  if (ctx->cg_part_cap < need) {
    cudaFree(ctx->cg_part);
    ctx->cg_part = nullptr;
    PSC_CUDA(ctx, cudaMalloc(&ctx->cg_part, 2 * (size_t)need * sizeof(double)));
    ctx->cg_part_cap = need;
  }
  if (!ctx->cg_x) PSC_CUDA(ctx, cudaMalloc(&ctx->cg_x, n * sizeof(double)));
  double* sc = ctx->scalars;
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->cg_x, x, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  // r = rhs - A x
  int rc = psc_laplacian_fused(ctx, ctx->cg_x, rhs, ctx->cg_r, -1.0, 0.0, 1.0, nullptr, nullptr, st);
  if (rc) return rc;
  const double* rr_a[1] = {ctx->cg_r};
  rc = psc_dots(ctx, 1, rr_a, rr_a, n, sc + 70, st);
  if (rc) return rc;
  k_cg_init<<<1, 32, 0, st>>>(sc, sc + 70, tol, maxit);
  PSC_LAUNCH_CHECK(ctx);
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->cg_p, ctx->cg_r, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  const bool use_graph = ctx->use_graphs;
  if (use_graph) {
    rc = cg_graph(ctx);
    if (rc) return rc;
  }
  for (int done = 0; done < maxit; done += CG_CHUNK) {
    if (use_graph) {
      PSC_CUDA(ctx, cudaGraphLaunch(ctx->cg_exec, st));
      // the graph's kernels are counted as launches too
      for (int i = 0; i < 3 * CG_CHUNK; ++i) psc_note_launch();
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

// 1: replay captured CUDA graphs for the CG iterations (default), 0: launch
// every kernel from the host.
extern "C" int psc_set_use_graphs(psc_ctx* ctx, int on) {
  if (!ctx) return 2;
  ctx->use_graphs = on ? 1 : 0;
  return 0;
}
