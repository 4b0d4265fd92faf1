// Persistent conjugate-gradient kernel for the Hartree solve
// (Eigensolvers/pcg.py:7-85), one cooperative launch per solve.
//
// The CG vectors of a whole grid fit in the shared memory of the GPU (a
// 78^3 grid needs 4 x 474,552 doubles = 15 MB against 148 x 227 KB), so each
// of G co-resident CTAs (one per SM) keeps x, r, p and Ap of a contiguous
// range [a, b) of flat grid points in shared memory for the entire solve.
// The only vector other CTAs read is r, mirrored to global memory after each
// update (read back with loads that bypass L1, since its owners rewrite it
// every iteration).
//
// Iteration it (same stop rule as the two-kernel CG in pcg.cu, including the
// reference's aliased first direction update):
//   A  s = A r: x and y neighbours from a shared-memory window of r over
//      [a - R nx, b + R nx), z neighbours straight from global r;
//      p = r + beta q and Ap = s + beta Aq with q = previous p (q = r in the
//      second iteration, p = r in the first) -- Ap by this recurrence rather
//      than a second stencil, the same quantity in exact arithmetic; partial
//      of p.Ap                                                 -> grid barrier
//   B  pAp from all partials (every CTA sums them in the same order), alpha,
//      x += alpha p, r -= alpha Ap; own r to global; partial of r.r
//                                                              -> grid barrier
//   C  ro1 from all partials; the stop decision and beta are then identical
//      in every CTA.
// The grid barrier is a monotone arrival counter with a bounded spin: a CTA
// that waits more than 4x the context's wait limit (2^26 polls by default)
// records status[4] and stops waiting, so a fault can never hang the GPU.  Every CTA takes the same number of barriers.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>

namespace {
constexpr int PNT = 1024;

__device__ __forceinline__ void grid_barrier(unsigned int* ctr, unsigned int target, int* status, bool& failed,
                                             long limit) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(ctr, 1u);
    if (!failed) {
      long spins = 0;
      while (true) {
        unsigned int v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(ctr) : "memory");
        if (v >= target) break;
        if (++spins > limit) {
          failed = true;
          atomicExch(&status[4], 1);
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// Sum of the G per-CTA partials part[0..G) by warp 0 in a fixed order, the
// same in every CTA; the result is broadcast through shared memory.
__device__ __forceinline__ double grid_sum(const double* part, int G, double* bc) {
  if (threadIdx.x < 32) {
    double s = 0.0;
    for (int t = threadIdx.x; t < G; t += 32) s += __ldcg(part + t);
    s = psc_warp_sum(s);
    if (threadIdx.x == 0) *bc = s;
  }
  __syncthreads();
  const double r = *bc;
  return r;
}
}  // namespace

template <int R>
__global__ void __launch_bounds__(PNT, 1)
k_cg_persistent(const double* __restrict__ rhs, double* __restrict__ xg, double* rg, int nx, int ny, int nz,
                double c0, double4 cw, int chunk, double* part, unsigned int* bar, int* status, double tol,
                int maxit, double* out, long bar_limit) {
  extern __shared__ double sm[];
  __shared__ double sh[PNT / 32];
  __shared__ double bc[2];
  __shared__ int s_failed;
  const int n = nx * ny * nz;
  const int nxy = nx * ny;
  const int G = gridDim.x;
  const int a = blockIdx.x * chunk;
  const int b = min(n, a + chunk);
  const int L = max(0, b - a);
  const int hw = R * nx;                 // window halo: the x and y neighbours
  const int W = chunk + 2 * hw;
  double* xs = sm;
  double* rs = sm + chunk;
  double* ps = sm + 2 * chunk;
  double* aps = sm + 3 * chunk;
  double* win = sm + 4 * chunk;          // win[w] = vector at flat a - hw + w (0 outside the grid)
  const double cd[4] = {cw.x, cw.y, cw.z, cw.w};
  unsigned int nbar = 0;
  bool failed = false;
  if (threadIdx.x == 0) s_failed = 0;

  // A v at own point t: x, y neighbours from the window, z neighbours from zsrc
  auto stencil = [&](int t, const double* zsrc) -> double {
    const int g = a + t;
    const int k = g / nxy;
    const int rem = g - k * nxy;
    const int j = rem / nx;
    const int i = rem - j * nx;
    const double* c = win + hw + t;
    double zv[2 * R];
#pragma unroll
    for (int d = 1; d <= R; ++d) {   // issue every z load before using any
      zv[2 * d - 2] = (k - d >= 0) ? __ldcg(zsrc + g - d * nxy) : 0.0;
      zv[2 * d - 1] = (k + d < nz) ? __ldcg(zsrc + g + d * nxy) : 0.0;
    }
    double acc = c0 * c[0];
#pragma unroll
    for (int d = 1; d <= R; ++d) {
      double s = zv[2 * d - 2] + zv[2 * d - 1];
      s += (i - d >= 0) ? c[-d] : 0.0;
      s += (i + d < nx) ? c[d] : 0.0;
      s += (j - d >= 0) ? c[-d * nx] : 0.0;
      s += (j + d < ny) ? c[d * nx] : 0.0;
      acc += cd[d - 1] * s;
    }
    return acc;
  };
  auto fill_window = [&](const double* own, const double* glob) {
    for (int w = threadIdx.x; w < W; w += PNT) {
      const int t = w - hw;
      const int g = a + t;
      double v = 0.0;
      if (t >= 0 && t < L) v = own[t];
      else if (g >= 0 && g < n) v = __ldcg(glob + g);
      win[w] = v;
    }
  };

  // ---- set-up: own x, r = rhs - A x, ro = r.r ----
  for (int t = threadIdx.x; t < L; t += PNT) xs[t] = xg[a + t];
  __syncthreads();
  fill_window(xs, xg);
  __syncthreads();
  double rr = 0.0;
  for (int t = threadIdx.x; t < L; t += PNT) {
    const double ri = rhs[a + t] - stencil(t, xg);
    rs[t] = ri;
    rg[a + t] = ri;
    rr += ri * ri;
  }
  rr = psc_block_sum<double, PNT>(rr, sh);
  if (threadIdx.x == 0) part[G + blockIdx.x] = rr;
  grid_barrier(bar, (++nbar) * G, status, failed, bar_limit);
  double ro = grid_sum(part + G, G, &bc[0]);
  const double tol1 = tol * tol * ro;
  int it = 0;
  bool active = maxit > 0 && ro > tol1;
  double beta = 0.0;
  while (active) {
    ++it;
    const bool alias = it <= 2;              // q = r in the first two iterations
    const double bt = it == 1 ? 0.0 : beta;  // p = r in the first
    // A: s = A r, direction, Ap, partial of p.Ap
    fill_window(rs, rg);
    __syncthreads();
    double pap = 0.0;
    for (int t = threadIdx.x; t < L; t += PNT) {
      const double sv = stencil(t, rg);
      const double rv = rs[t];
      const double pv = rv + bt * (alias ? rv : ps[t]);
      const double av = sv + bt * (alias ? sv : aps[t]);
      ps[t] = pv;
      aps[t] = av;
      pap += av * pv;
    }
    pap = psc_block_sum<double, PNT>(pap, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = pap;
    grid_barrier(bar, (++nbar) * G, status, failed, bar_limit);
    pap = grid_sum(part, G, &bc[0]);
    // B: alpha, updates, partial of r.r
    const double alp = ro / pap;
    rr = 0.0;
    for (int t = threadIdx.x; t < L; t += PNT) {
      xs[t] += alp * ps[t];
      const double ri = rs[t] - alp * aps[t];
      rs[t] = ri;
      rg[a + t] = ri;
      rr += ri * ri;
    }
    rr = psc_block_sum<double, PNT>(rr, sh);
    if (threadIdx.x == 0) part[G + blockIdx.x] = rr;
    grid_barrier(bar, (++nbar) * G, status, failed, bar_limit);
    // C: stop test and beta, identical in every CTA
    const double ro1 = grid_sum(part + G, G, &bc[1]);
    beta = ro1 / ro;
    ro = ro1;
    active = it < maxit && ro1 > tol1;
    if (threadIdx.x == 0 && failed) s_failed = 1;
    __syncthreads();
    if (s_failed) active = false;  // a barrier gave up: leave in step
  }
  for (int t = threadIdx.x; t < L; t += PNT) xg[a + t] = xs[t];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    out[0] = (double)it;
    out[1] = ro;
  }
}

// Persistent solve if the vectors fit in shared memory; returns -1 if not
// (the caller then uses the graph-replayed kernels).
int psc_pcg_persistent(psc_ctx* ctx, const double* rhs, double* x, int maxit, double tol, int* its_out,
                       cudaStream_t st) {
  if (ctx->cg_persistent == 0) return -1;
  int sms = 0, dev = ctx->device;
  PSC_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int coop = 0;
  PSC_CUDA(ctx, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  if (!coop || sms <= 0) return -1;
  const long n = ctx->n;
  if (n >= (1L << 31) - 1) return -1;
  const int G = sms;
  const int R = ctx->radius;
  const long chunk = (n + G - 1) / G;
  const size_t smem = (5 * (size_t)chunk + 2 * (size_t)R * ctx->nx) * sizeof(double);
  int optin = 0;
  PSC_CUDA(ctx, cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (smem + 2048 > (size_t)optin) return -1;
  void* fn = nullptr;
  switch (R) {
    case 1: fn = (void*)k_cg_persistent<1>; break;
    case 2: fn = (void*)k_cg_persistent<2>; break;
    case 3: fn = (void*)k_cg_persistent<3>; break;
    default: fn = (void*)k_cg_persistent<4>; break;
  }
  PSC_CUDA(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  PSC_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, PNT, smem));
  if (per_sm < 1) return -1;
  if (!ctx->cg_r) PSC_CUDA(ctx, psc_dmalloc(&ctx->cg_r, n * sizeof(double)));
  if (!ctx->cg_bar) PSC_CUDA(ctx, psc_dmalloc(&ctx->cg_bar, 64 * sizeof(unsigned int)));
  if (ctx->cg_part_cap < G) {
    psc_dfree(ctx->cg_part);
    ctx->cg_part = nullptr;
    PSC_CUDA(ctx, psc_dmalloc(&ctx->cg_part, 2 * (size_t)std::max(G, PSC_RED_BLOCKS) * sizeof(double)));
    ctx->cg_part_cap = std::max(G, PSC_RED_BLOCKS);
  }
  PSC_CUDA(ctx, cudaMemsetAsync(ctx->cg_bar, 0, 64 * sizeof(unsigned int), st));
  const double4 cw = make_double4(ctx->lap_c[0], ctx->lap_c[1], ctx->lap_c[2], ctx->lap_c[3]);
  double* out = ctx->scalars + 80;
  double* rg = ctx->cg_r;
  unsigned int* bar = ctx->cg_bar;
  int* status = ctx->dev_status;
  int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
  double c0 = ctx->lap_c0;
  int chunk_i = (int)chunk;
  double* part = ctx->cg_part;
  long bar_limit = 4 * ctx->wait_limit;   // grid barriers wait 4x longer than the mbarrier pipelines
  void* args[] = {(void*)&rhs, (void*)&x, (void*)&rg, (void*)&nx, (void*)&ny, (void*)&nz, (void*)&c0, (void*)&cw,
                  (void*)&chunk_i, (void*)&part, (void*)&bar, (void*)&status, (void*)&tol, (void*)&maxit, (void*)&out,
                  (void*)&bar_limit};
  PSC_CUDA(ctx, cudaLaunchCooperativeKernel(fn, dim3(G), dim3(PNT), args, smem, st));
  PSC_LAUNCH_CHECK(ctx);
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->host_scalars + 80, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  int* hflag = reinterpret_cast<int*>(ctx->host_scalars + 82);
  PSC_CUDA(ctx, cudaMemcpyAsync(hflag, status + 4, sizeof(int), cudaMemcpyDeviceToHost, st));
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  if (*hflag) {
    psc_set_error(ctx, "pcg: persistent CG grid barrier timed out (CTAs not co-resident?)");
    return 1;
  }
  if (its_out) *its_out = (int)ctx->host_scalars[80];
  return 0;
}
