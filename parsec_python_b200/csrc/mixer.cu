// Multisecant Type-I potential mixing with group size 1 (Broyden's first
// method): Mixer/msecant1.py:40-175 with the parameters of
// Mixer/includemix.py:21-49 (mix 0.5, restart factor 0.1, EN_like 0).
//
// The secant history DX, DF (one n-vector per SCF iteration) stays in HBM.
// A call reads the history twice: once for the 3(m-1) dot products
// DF_i.df, DF_i.f1, DX_i.dx and once to form the new DX column, the new
// iterate and the group vector N.  The 1x1 quasi-inverse of
// Mixer/qinv.py:5-62 is 1/M (0 when M == 0).
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <cmath>

__global__ void k_mix_first(const double* __restrict__ x1, const double* __restrict__ f1, double mix, long n,
                            double* __restrict__ dx0, double* __restrict__ df0, double* __restrict__ xn) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    dx0[i] = x1[i];
    df0[i] = f1[i];
    xn[i] = x1[i] + mix * f1[i];
  }
}

__global__ void k_mix_restart(const double* __restrict__ xl, const double* __restrict__ fl, double mix, long n,
                              double* __restrict__ dx0, double* __restrict__ df0, double* __restrict__ xn) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double x = xl[i], f = fl[i];
    xn[i] = x + mix * f;
    dx0[i] = x;
    df0[i] = f;
  }
}

// dx = x1 - DX[m-1], df = f1 - DF[m-1]; DF[m-1] <- df; tmp <- dx
__global__ void k_mix_diff(const double* __restrict__ x1, const double* __restrict__ f1, double* __restrict__ dxl,
                           double* __restrict__ dfl, double* __restrict__ tmp, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    tmp[i] = x1[i] - dxl[i];
    dfl[i] = f1[i] - dfl[i];
  }
}

// partials of a_i = DF_i.df, b_i = DF_i.f1, c_i = DX_i.dx for i < mm
__global__ void __launch_bounds__(256)
k_mix_dots(const double* __restrict__ DX, const double* __restrict__ DF, const double* __restrict__ df,
           const double* __restrict__ f1, const double* __restrict__ dx, long n, int mm, double* __restrict__ part) {
  __shared__ double sh[8];
  const long chunk = (n + gridDim.x - 1) / gridDim.x;
  const long lo = chunk * blockIdx.x, hi = min(n, lo + chunk);
  for (int i = 0; i < mm; ++i) {
    const double* dfi = DF + (long)i * n;
    const double* dxi = DX + (long)i * n;
    double a = 0.0, b = 0.0, c = 0.0;
    for (long p = lo + threadIdx.x; p < hi; p += 256) {
      const double v = dfi[p];
      a += v * df[p];
      b += v * f1[p];
      c += dxi[p] * dx[p];
    }
    a = psc_block_sum<double, 256>(a, sh);
    if (threadIdx.x == 0) part[(long)(3 * i + 0) * PSC_RED_BLOCKS + blockIdx.x] = a;
    b = psc_block_sum<double, 256>(b, sh);
    if (threadIdx.x == 0) part[(long)(3 * i + 1) * PSC_RED_BLOCKS + blockIdx.x] = b;
    c = psc_block_sum<double, 256>(c, sh);
    if (threadIdx.x == 0) part[(long)(3 * i + 2) * PSC_RED_BLOCKS + blockIdx.x] = c;
  }
}

__global__ void k_mix_reduce(const double* __restrict__ part, int nslots, double* __restrict__ out) {
  __shared__ double sh[8];
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    double v = 0.0;
    for (int i = threadIdx.x; i < PSC_RED_BLOCKS; i += 256) v += part[(long)s * PSC_RED_BLOCKS + i];
    v = psc_block_sum<double, 256>(v, sh);
    if (threadIdx.x == 0) out[s] = v;
  }
}

// DX[m-1] = dx + mix df - sum DX_i a_i ; xn = x1 + mix f1 - sum DX_i b_i ;
// N = -mix dx + sum DF_i c_i ; partials of N.df and N.f1
__global__ void __launch_bounds__(256)
k_mix_combine(double* __restrict__ DX, const double* __restrict__ DF, const double* __restrict__ x1,
              const double* __restrict__ f1, const double* __restrict__ dx, long n, int m, double mix,
              const double* __restrict__ coef, double* __restrict__ xn, double* __restrict__ nv,
              double* __restrict__ part) {
  __shared__ double sh[8];
  __shared__ double cf[3 * 256];
  const int mm = m - 1;
  for (int i = threadIdx.x; i < 3 * mm; i += 256) cf[i] = coef[i];
  __syncthreads();
  const double* df = DF + (long)mm * n;
  double* dxl = DX + (long)mm * n;
  double s0 = 0.0, s1 = 0.0;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    const double dxp = dx[p], dfp = df[p];
    double d = dxp + mix * dfp;
    double x = x1[p] + mix * f1[p];
    double nn = -mix * dxp;
    for (int i = 0; i < mm; ++i) {
      const double hx = DX[(long)i * n + p];
      d -= hx * cf[3 * i + 0];
      x -= hx * cf[3 * i + 1];
      nn += DF[(long)i * n + p] * cf[3 * i + 2];
    }
    dxl[p] = d;
    xn[p] = x;
    nv[p] = nn;
    s0 += nn * dfp;
    s1 += nn * f1[p];
  }
  s0 = psc_block_sum<double, 256>(s0, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s0;
  s1 = psc_block_sum<double, 256>(s1, sh);
  if (threadIdx.x == 0) part[PSC_RED_BLOCKS + blockIdx.x] = s1;
}

// C = qinv([M]) = 1/M (0 when M == 0); DF[m-1] = N C; xn -= DX[m-1] * (C * N.f1);
// append DX[m] = x1, DF[m] = f1
__global__ void k_mix_final(double* __restrict__ DX, double* __restrict__ DF, const double* __restrict__ x1,
                            const double* __restrict__ f1, const double* __restrict__ nv, long n, int m,
                            const double* __restrict__ s /* [M, N.f1] */, double* __restrict__ xn) {
  const double M = s[0];
  const double C = (M != 0.0) ? 1.0 / M : 0.0;
  const double g = C * s[1];
  double* dfl = DF + (long)(m - 1) * n;
  const double* dxl = DX + (long)(m - 1) * n;
  double* dxa = DX + (long)m * n;
  double* dfa = DF + (long)m * n;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    dfl[p] = nv[p] * C;
    xn[p] -= dxl[p] * g;
    dxa[p] = x1[p];
    dfa[p] = f1[p];
  }
}

extern "C" int psc_mixer_reset(psc_ctx* ctx, int capacity) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, capacity >= 1 && capacity <= 255, "mixer: capacity must be 1..255");
  if (capacity > ctx->mix_cap) {
    psc_dfree(ctx->mix_dx); psc_dfree(ctx->mix_df); psc_dfree(ctx->mix_nv); psc_dfree(ctx->mix_tmp);
    psc_dfree(ctx->mix_coef); psc_dfree(ctx->mix_partial);
    ctx->mix_dx = ctx->mix_df = ctx->mix_nv = ctx->mix_tmp = ctx->mix_coef = ctx->mix_partial = nullptr;
    const size_t n = ctx->n;
    PSC_CUDA(ctx, psc_dmalloc(&ctx->mix_dx, (size_t)(capacity + 1) * n * sizeof(double)));
    PSC_CUDA(ctx, psc_dmalloc(&ctx->mix_df, (size_t)(capacity + 1) * n * sizeof(double)));
    PSC_CUDA(ctx, psc_dmalloc(&ctx->mix_nv, n * sizeof(double)));
    PSC_CUDA(ctx, psc_dmalloc(&ctx->mix_tmp, n * sizeof(double)));
    PSC_CUDA(ctx, psc_dmalloc(&ctx->mix_coef, (3 * (size_t)capacity + 8) * sizeof(double)));
    PSC_CUDA(ctx, psc_dmalloc(&ctx->mix_partial, (3 * (size_t)capacity + 2) * PSC_RED_BLOCKS * sizeof(double)));
    ctx->mix_cap = capacity;
  }
  ctx->mix_m = 0;
  ctx->mix_last_fnorm = -1.0;
  return 0;
}

// x_new = mixer(x1, f1).  *m_used receives the number of secant equations
// (0 for the first call and after a restart), as Mixer/mixer.py:189-217.
extern "C" int psc_mixer_step(psc_ctx* ctx, const double* x1, const double* f1, double mix, double restart_factor,
                              double* x_new, int* m_used, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, ctx->mix_cap > 0, "mixer: call psc_mixer_reset first");
  PSC_REQUIRE(ctx, x_new != x1 && x_new != f1, "mixer: output must not alias the inputs");
  cudaStream_t st = (cudaStream_t)stream;
  const long n = ctx->n;
  const int nb = PSC_RED_BLOCKS;
  const int m = ctx->mix_m;
  // |f1| for the restart test and for the next call
  const double* fa[1] = {f1};
  int rc = psc_dots(ctx, 1, fa, fa, n, ctx->scalars + 120, st);
  if (rc) return rc;
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->host_scalars + 120, ctx->scalars + 120, sizeof(double), cudaMemcpyDeviceToHost, st));
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  const double fnorm = std::sqrt(ctx->host_scalars[120]);
  if (m == 0) {
    k_mix_first<<<nb, 256, 0, st>>>(x1, f1, mix, n, ctx->mix_dx, ctx->mix_df, x_new);
    PSC_LAUNCH_CHECK(ctx);
    ctx->mix_m = 1;
    ctx->mix_last_fnorm = fnorm;
    if (m_used) *m_used = 0;
    return 0;
  }
  if (m >= 2 && ctx->mix_last_fnorm < restart_factor * fnorm) {
    k_mix_restart<<<nb, 256, 0, st>>>(ctx->mix_dx + (long)(m - 1) * n, ctx->mix_df + (long)(m - 1) * n, mix, n,
                                      ctx->mix_dx, ctx->mix_df, x_new);
    PSC_LAUNCH_CHECK(ctx);
    ctx->mix_m = 1;
    if (m_used) *m_used = 0;
    return 0;
  }
  PSC_REQUIRE(ctx, m + 1 <= ctx->mix_cap, "mixer: history capacity exceeded (raise it at reset)");
  double* dxl = ctx->mix_dx + (long)(m - 1) * n;
  double* dfl = ctx->mix_df + (long)(m - 1) * n;
  k_mix_diff<<<nb, 256, 0, st>>>(x1, f1, dxl, dfl, ctx->mix_tmp, n);
  PSC_LAUNCH_CHECK(ctx);
  const int mm = m - 1;
  if (mm > 0) {
    k_mix_dots<<<nb, 256, 0, st>>>(ctx->mix_dx, ctx->mix_df, dfl, f1, ctx->mix_tmp, n, mm, ctx->mix_partial);
    PSC_LAUNCH_CHECK(ctx);
    k_mix_reduce<<<std::min(3 * mm, 148), 256, 0, st>>>(ctx->mix_partial, 3 * mm, ctx->mix_coef);
    PSC_LAUNCH_CHECK(ctx);
  }
  k_mix_combine<<<nb, 256, 0, st>>>(ctx->mix_dx, ctx->mix_df, x1, f1, ctx->mix_tmp, n, m, mix, ctx->mix_coef, x_new,
                                    ctx->mix_nv, ctx->mix_partial);
  PSC_LAUNCH_CHECK(ctx);
  double* sv = ctx->mix_coef + 3 * ctx->mix_cap;
  k_mix_reduce<<<2, 256, 0, st>>>(ctx->mix_partial, 2, sv);
  PSC_LAUNCH_CHECK(ctx);
  k_mix_final<<<nb, 256, 0, st>>>(ctx->mix_dx, ctx->mix_df, x1, f1, ctx->mix_nv, n, m, sv, x_new);
  PSC_LAUNCH_CHECK(ctx);
  ctx->mix_m = m + 1;
  ctx->mix_last_fnorm = fnorm;
  if (m_used) *m_used = m;
  return 0;
}

extern "C" int psc_mixer_history(psc_ctx* ctx, int* m_out) {
  if (!ctx) return 2;
  if (m_out) *m_out = ctx->mix_m;
  return 0;
}
