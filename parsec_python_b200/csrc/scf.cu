// Per-iteration SCF kernels: Lanczos spectrum bounds, Fermi-Dirac
// occupations, electron density, LDA exchange-correlation and the potential
// update with its error and energy sums.  Scalars stay on the device; the
// host reads one small block per SCF iteration.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>
#include <cmath>

// ---------------------------------------------------------------------------
// vector helpers on device scalars
// ---------------------------------------------------------------------------
// y = x / s[0]
__global__ void k_scale_by(const double* __restrict__ x, double* __restrict__ y, long n, const double* s) {
  const double d = *s;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) y[i] = x[i] / d;
}
// y -= s[0] * x
__global__ void k_axpy_neg(const double* __restrict__ x, double* __restrict__ y, long n, const double* s) {
  const double a = *s;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) y[i] = y[i] - a * x[i];
}

// Lanczos scalar bookkeeping.  sc layout (device):
//  [0] alpha  [1] beta  [2] dot scratch  [8..8+6] alphas  [16..16+6] betas
__global__ void k_lz_sqrt_beta(double* sc, int rescale, int j) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double b = sqrt(sc[2]);
    if (rescale && b < 1e-2) b = b * 10;  // lancz_uppbnd.py:65-66
    sc[1] = b;
    sc[16 + j] = b;
  }
}
__global__ void k_lz_store_alpha(double* sc, int j) {
  if (threadIdx.x == 0 && blockIdx.x == 0) sc[8 + j] = sc[0];
}
__global__ void k_lz_tridiag(const double* sc, int m, double* T) {
  // dense m x m tridiagonal: diag alphas, off-diagonal betas[0..m-2]
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
    const int i = e % m, j = e / m;
    double v = 0.0;
    if (i == j) v = sc[8 + i];
    else if (i == j + 1 || j == i + 1) v = sc[16 + min(i, j)];
    T[e] = v;
  }
}
// mode 0 (lancz_uppbnd.py:68-75): out = [uppbnd, ritz_0..ritz_{m-1}]
// mode 1 (lanczosForChefsi1.py:164): out = [max|ritz| + beta_m]
__global__ void k_lz_bound(const double* sc, int m, const double* ritz, const double* X, int mode, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double beta = sc[16 + m - 1];
  if (mode == 0) {
    const double top = ritz[m - 1];
    const double u0 = top + beta;
    const double u1 = top + fabs(X[(m - 1) + (long)(m - 1) * m]) * beta;
    double mx = 0.0;
    for (int j = 0; j < m; ++j) mx = fmax(mx, fabs(X[(m - 1) + (long)j * m]));
    const double u2 = top + mx * beta;
    double ub = (u0 + u1) / 2;
    ub = (u2 + ub) / 2;
    out[0] = ub;
    for (int j = 0; j < m; ++j) out[1 + j] = ritz[j];
  } else {
    double mx = 0.0;
    for (int j = 0; j < m; ++j) mx = fmax(mx, fabs(ritz[j]));
    out[0] = mx + beta;
  }
}

// Six-step Lanczos estimate of the top of the spectrum of H (FP64).
//   mode 0: lancz_uppbnd (Eigensolvers/lancz_uppbnd.py:4-75): uniform start,
//           out = [uppbnd, ritz_0..ritz_5] (ritz ascending)
//   mode 1: lanczosForChefsi1 (Eigensolvers/lanczosForChefsi1.py:5-99):
//           normal start, out = [max|ritz| + beta_6]
int psc_lanczos_bound_basis(psc_ctx* ctx, unsigned long long seed, const double* v_start, double* out_dev,
                            cudaStream_t st);

// The six-step bounds; v_start (device, n, may be NULL) replaces the vector
// drawn from `seed` (the reference draws np.random.rand for lancz_uppbnd and
// np.random.randn for chefsi1's lanczosForChefsi1).
static int lanczos_bound_impl(psc_ctx* ctx, int mode, unsigned long long seed, const double* v_start,
                              double* out_dev, cudaStream_t st) {
  // mode 1 runs the three-term recurrence of psc_lanczos_run (the same steps,
  // fused, keeping a basis of 7 vectors) and bisection on T_6
  if (mode != 0) return psc_lanczos_bound_basis(ctx, seed, v_start, out_dev, st);
  const long n = ctx->n;
  const int m = 6;
  if (psc_ensure_dense(ctx, m)) return 1;
  double* v0 = ctx->lz_v;
  double* v = ctx->lz_v + n;
  double* f = ctx->lz_v + 2 * n;
  double* sc = ctx->scalars;  // [0..31]
  const int nb = 148 * 8;
  int rc = 0;
  if (v_start) {
    PSC_CUDA(ctx, cudaMemcpyAsync(f, v_start, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  } else {
    rc = psc_random_impl(ctx, PSC_F64, mode == 0 ? 0 : 1, seed, f, n, n, 1, st);
    if (rc) return rc;
  }
  // v = f / ||f||
  const double* a1[1] = {f};
  rc = psc_dots(ctx, 1, a1, a1, n, sc + 2, st);
  if (rc) return rc;
  k_lz_sqrt_beta<<<1, 32, 0, st>>>(sc, 0, 31);  // sc[1] = ||f||  (slot 16+31 unused)
  PSC_LAUNCH_CHECK(ctx);
  k_scale_by<<<nb, 256, 0, st>>>(f, v, n, sc + 1);
  PSC_LAUNCH_CHECK(ctx);
  if (mode == 0) {
    // f = H v; alpha = v.f; f -= alpha v; T[0,0] = alpha; beta = ||f||
    rc = psc_apply_h_impl(ctx, PSC_F64, v, n, f, n, nullptr, 0, 1, nullptr, 1.0, 0.0, 0.0, st);
    if (rc) return rc;
    const double* da[1] = {v};
    const double* db[1] = {f};
    rc = psc_dots(ctx, 1, da, db, n, sc + 0, st);
    if (rc) return rc;
    k_axpy_neg<<<nb, 256, 0, st>>>(v, f, n, sc + 0);
    PSC_LAUNCH_CHECK(ctx);
    k_lz_store_alpha<<<1, 32, 0, st>>>(sc, 0);
    PSC_LAUNCH_CHECK(ctx);
    rc = psc_dots(ctx, 1, a1, a1, n, sc + 2, st);
    if (rc) return rc;
    k_lz_sqrt_beta<<<1, 32, 0, st>>>(sc, 0, 0);  // first beta, no rescale
    PSC_LAUNCH_CHECK(ctx);
    for (int j = 1; j < m; ++j) {
      // v0 = v; v = f/beta; f = H v - beta v0; alpha = v.f; f -= alpha v; beta = ||f||
      std::swap(v0, v);
      k_scale_by<<<nb, 256, 0, st>>>(f, v, n, sc + 1);
      PSC_LAUNCH_CHECK(ctx);
      rc = psc_apply_h_impl(ctx, PSC_F64, v, n, f, n, nullptr, 0, 1, nullptr, 1.0, 0.0, 0.0, st);
      if (rc) return rc;
      k_axpy_neg<<<nb, 256, 0, st>>>(v0, f, n, sc + 1);
      PSC_LAUNCH_CHECK(ctx);
      const double* va[1] = {v};
      const double* fb[1] = {f};
      rc = psc_dots(ctx, 1, va, fb, n, sc + 0, st);
      if (rc) return rc;
      k_axpy_neg<<<nb, 256, 0, st>>>(v, f, n, sc + 0);
      PSC_LAUNCH_CHECK(ctx);
      k_lz_store_alpha<<<1, 32, 0, st>>>(sc, j);
      PSC_LAUNCH_CHECK(ctx);
      rc = psc_dots(ctx, 1, a1, a1, n, sc + 2, st);
      if (rc) return rc;
      k_lz_sqrt_beta<<<1, 32, 0, st>>>(sc, 1, j);
      PSC_LAUNCH_CHECK(ctx);
    }
    // betas used in T are the ones preceding each step: T[j,j-1] = beta_{j-1}
    k_lz_tridiag<<<1, 64, 0, st>>>(sc, m, ctx->gram);
    PSC_LAUNCH_CHECK(ctx);
    rc = psc_syev_impl(ctx, ctx->gram, m, sc + 40, ctx->evec, st);
    if (rc) return rc;
    k_lz_bound<<<1, 32, 0, st>>>(sc, m, sc + 40, ctx->evec, 0, out_dev);
    PSC_LAUNCH_CHECK(ctx);
  }
  return 0;
}

extern "C" int psc_lanczos_bound(psc_ctx* ctx, int mode, unsigned long long seed, double* out_dev, void* stream) {
  if (!ctx) return 2;
  return lanczos_bound_impl(ctx, mode, seed, nullptr, out_dev, (cudaStream_t)stream);
}

extern "C" int psc_lanczos_bound_v(psc_ctx* ctx, int mode, const double* v_start, double* out_dev, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, v_start && out_dev, "lanczos_bound_v: NULL pointer argument");
  return lanczos_bound_impl(ctx, mode, 0, v_start, out_dev, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// filter bounds from device values
// ---------------------------------------------------------------------------
// mode 0 (chefsi1.py:29-38): bounds = [min(ritz), max(ritz), upper]
// mode 1 (first_filt.py:28-29): bounds = [0, 0.8*r6[0] + 0.2*r6[4], upper]
// mode 2 (first_filt.py:62):    bounds = [0, max(ritz), upper]
__global__ void k_bounds(int mode, const double* ritz, int k, const double* upper, double* bounds) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (mode == 0) {
    double lo = ritz[0], hi = ritz[0];
    for (int i = 1; i < k; ++i) { lo = fmin(lo, ritz[i]); hi = fmax(hi, ritz[i]); }
    bounds[0] = lo; bounds[1] = hi; bounds[2] = upper[0];
  } else if (mode == 1) {
    bounds[0] = 0.0; bounds[1] = 0.8 * ritz[0] + 0.2 * ritz[4]; bounds[2] = upper[0];
  } else {
    bounds[0] = 0.0; bounds[1] = ritz[k - 1]; bounds[2] = upper[0];
  }
}

extern "C" int psc_filter_bounds(psc_ctx* ctx, int mode, const double* ritz_dev, int k, const double* upper_dev,
                                 double* bounds_dev, void* stream) {
  if (!ctx) return 2;
  k_bounds<<<1, 32, 0, (cudaStream_t)stream>>>(mode, ritz_dev, k, upper_dev, bounds_dev);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

// ---------------------------------------------------------------------------
// occupations: bisection for the Fermi level (Eigensolvers/occupations.py:5-56,
// Eigensolvers/FermiDirac.py:3-31), one warp.
// ---------------------------------------------------------------------------
__device__ double fd_sum(const double* lam, int n, double ef, double kT, double* occ) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += 32) {
    const double lg = (lam[i] - ef) / kT;
    const double e = exp(-fabs(lg));
    const double o = lg >= 0 ? e / (1.0 + e) : 1.0 / (1.0 + e);
    if (occ) occ[i] = o;
    s += o;
  }
  return psc_warp_sum(s);
}

__global__ void k_occupations(const double* __restrict__ lam, int n, double temp, double nelec, double tol,
                              double* __restrict__ ef_out, double* __restrict__ occ) {
  const double kT = temp * 6.33327186e-06;
  double lmin = 1e300;
  for (int i = threadIdx.x; i < n; i += 32) lmin = fmin(lmin, lam[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lmin = fmin(lmin, __shfl_xor_sync(0xffffffffu, lmin, o));
  double a = lmin - 1;
  const double fa = fd_sum(lam, n, a, kT, nullptr) - nelec / 2;
  const int lmax = min(max(1, (int)ceil(nelec / 2) + 1), n);
  double b = lam[lmax - 1] + 1;
  double fb = fd_sum(lam, n, b, kT, nullptr) - nelec / 2;
  double c = (b + a) / 2;
  double err = 2 * fd_sum(lam, n, c, kT, occ) - nelec;
  if (fa * fb > tol) {
    for (int i = threadIdx.x; i < n; i += 32) occ[i] = 1.0;
    if (threadIdx.x == 0) *ef_out = b;
    return;
  }
  int its = 0;
  while (fabs(err) > tol && its < 200) {
    ++its;
    c = (b + a) / 2;
    __syncwarp();
    const double s = fd_sum(lam, n, c, kT, occ);
    const double fc = s - nelec / 2;
    err = 2 * s - nelec;
    if (fc * fb < 0) a = c;
    else { b = c; fb = fc; }
  }
  if (threadIdx.x == 0) *ef_out = c;
}

extern "C" int psc_occupations(psc_ctx* ctx, const double* lam_dev, int n, double temp, double nelec, double tol,
                               double* ef_dev, double* occ_dev, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, n >= 1, "occupations: empty eigenvalue list");
  k_occupations<<<1, 32, 0, (cudaStream_t)stream>>>(lam_dev, n, temp, nelec, tol, ef_dev, occ_dev);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

// ---------------------------------------------------------------------------
// density: rho_raw = sum_i W_i^2 (2 f_i) (rsdft_solver.py:324),
// hrhs = 4pi/h^3 (rho_raw - rho0), rho = rho_raw / h^3 (rsdft_solver.py:327-328)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_density(const T* __restrict__ W, long ld, int nev, const double* __restrict__ wgt,
                          const double* __restrict__ rho0, double* __restrict__ rho, double* __restrict__ hrhs, long n,
                          double fourpi_h3, double h3) {
  __shared__ double f2[1024];
  for (int i = threadIdx.x; i < nev; i += blockDim.x) f2[i] = wgt[i];
  __syncthreads();
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < nev; ++i) {
      const double w = (double)W[p + (long)i * ld];
      s += w * w * f2[i];
    }
    if (hrhs) hrhs[p] = fourpi_h3 * (s - rho0[p]);
    rho[p] = s / h3;
  }
}

// the density weight of each state, 2 occ_i, divided for FP32 blocks by the
// state's exact squared norm (its PSC_NORM_CHUNKS partials summed in order);
// formed once per call instead of in every block of k_density
__global__ void k_density_weights(const double* __restrict__ occ, const double* __restrict__ norm_part, int nev,
                                  double* __restrict__ wgt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nev; i += gridDim.x * blockDim.x) {
    double w = 2 * occ[i];
    if (norm_part) {
      double nn = 0.0;
      for (int c = 0; c < PSC_NORM_CHUNKS; ++c) nn += norm_part[(long)i * PSC_NORM_CHUNKS + c];
      w /= nn;
    }
    wgt[i] = w;
  }
}

// Exact FP64 squared norms of the columns of an FP32 block, as
// PSC_NORM_CHUNKS partial sums per column (summed in a fixed order by the
// consumer).  FP32 blocks carry a small column-scale error (the tensor cores'
// FP32 accumulation rounds toward zero, FP32 storage rounds each entry);
// the density divides each orbital's weight by its measured norm so that the
// electron count stays exact.
__global__ void __launch_bounds__(256)
k_colnorm_part(const float* __restrict__ W, long ld, long n, long chunk, double* __restrict__ part) {
  __shared__ double sh[8];
  const int col = blockIdx.y;
  const long r0 = (long)blockIdx.x * chunk;
  const long r1 = min(n, r0 + chunk);
  const float* w = W + (long)col * ld;
  double s = 0.0;
  for (long p = r0 + threadIdx.x; p < r1; p += 256) {
    const double v = (double)w[p];
    s = fma(v, v, s);
  }
  s = psc_block_sum<double, 256>(s, sh);
  if (threadIdx.x == 0) part[(long)col * PSC_NORM_CHUNKS + blockIdx.x] = s;
}

extern "C" int psc_density(psc_ctx* ctx, int dtype, const void* W, long ld, int nev, const double* occ_dev,
                           const double* rho0, double fourpi_h3, double h3, double* rho, double* hrhs,
                           void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, nev >= 1 && nev <= 1024, "density: nev out of range");
  PSC_REQUIRE(ctx, W && occ_dev && rho && ld >= ctx->n && (!hrhs || rho0), "density: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = 148 * 8;
  if (!ctx->dens_w) PSC_CUDA(ctx, psc_dmalloc(&ctx->dens_w, 1024 * sizeof(double)));
  if (dtype == PSC_F64) {
    k_density_weights<<<1, 1024, 0, st>>>(occ_dev, nullptr, nev, ctx->dens_w);
    PSC_LAUNCH_CHECK(ctx);
    k_density<double><<<nb, 256, 0, st>>>((const double*)W, ld, nev, ctx->dens_w, rho0, rho, hrhs, ctx->n,
                                          fourpi_h3, h3);
  } else {
    if (ctx->col_norm_cap < nev) {
      psc_dfree(ctx->col_norm_part);
      ctx->col_norm_part = nullptr;
      ctx->col_norm_cap = 0;
      PSC_CUDA(ctx, psc_dmalloc(&ctx->col_norm_part, (size_t)1024 * PSC_NORM_CHUNKS * sizeof(double)));
      ctx->col_norm_cap = 1024;
    }
    const long chunk = (ctx->n + PSC_NORM_CHUNKS - 1) / PSC_NORM_CHUNKS;
    k_colnorm_part<<<dim3(PSC_NORM_CHUNKS, nev), 256, 0, st>>>((const float*)W, ld, ctx->n, chunk,
                                                               ctx->col_norm_part);
    PSC_LAUNCH_CHECK(ctx);
    k_density_weights<<<1, 1024, 0, st>>>(occ_dev, ctx->col_norm_part, nev, ctx->dens_w);
    PSC_LAUNCH_CHECK(ctx);
    k_density<float><<<nb, 256, 0, st>>>((const float*)W, ld, nev, ctx->dens_w, rho0, rho, hrhs, ctx->n,
                                         fourpi_h3, h3);
  }
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

// ---------------------------------------------------------------------------
// LDA exchange-correlation (V_xc/exc_nspn.py:8-103), Ry units.
// out_dev = [exc (h^3 * sum), max rho, min rho]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_xc(const double* __restrict__ rho, double* __restrict__ vxc, long n, double* __restrict__ partial) {
  __shared__ double sh[8];
  double e = 0.0, mx = -1e300, mn = 1e300;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double r = rho[i];
    mx = psc_nanmax(mx, r);
    mn = psc_nanmin(mn, r);
    vxc[i] = psc_lda_point(r, e);
  }
  e = psc_block_sum<double, 256>(e, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = e;
  // max / min via warp shuffles and shared memory
  __shared__ double smx[8], smn[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = psc_nanmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mn = psc_nanmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  }
  if ((threadIdx.x & 31) == 0) { smx[threadIdx.x >> 5] = mx; smn[threadIdx.x >> 5] = mn; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; ++w) { mx = psc_nanmax(mx, smx[w]); mn = psc_nanmin(mn, smn[w]); }
    partial[PSC_RED_BLOCKS + blockIdx.x] = mx;
    partial[2 * PSC_RED_BLOCKS + blockIdx.x] = mn;
  }
}

__global__ void k_xc_final(const double* partial, double h3, double* out) {
  __shared__ double sh[8];
  double s = 0.0;
  for (int i = threadIdx.x; i < PSC_RED_BLOCKS; i += 256) s += partial[i];
  s = psc_block_sum<double, 256>(s, sh);
  if (threadIdx.x == 0) {
    double mx = -1e300, mn = 1e300;
    for (int i = 0; i < PSC_RED_BLOCKS; ++i) {
      mx = psc_nanmax(mx, partial[PSC_RED_BLOCKS + i]);
      mn = psc_nanmin(mn, partial[2 * PSC_RED_BLOCKS + i]);
    }
    out[0] = s * h3;
    out[1] = mx;
    out[2] = mn;
  }
}

extern "C" int psc_lda_xc(psc_ctx* ctx, const double* rho, double* vxc, double h3, double* out_dev, void* stream) {
  if (!ctx) {
    psc_set_error(nullptr, "psc_lda_xc: NULL context");
    return 2;
  }
  PSC_REQUIRE(ctx, rho && vxc && out_dev, "psc_lda_xc: NULL pointer argument");
  cudaStream_t st = (cudaStream_t)stream;
  k_xc<<<PSC_RED_BLOCKS, 256, 0, st>>>(rho, vxc, ctx->n, ctx->red_partial);
  PSC_LAUNCH_CHECK(ctx);
  k_xc_final<<<1, 256, 0, st>>>(ctx->red_partial, h3, out_dev);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

// ---------------------------------------------------------------------------
// potential update (rsdft_solver.py:351-352) and energy sums (:141-146)
//   pot_new = ppot + 0.5*vxc + hpot + hpot0 ; f = pot_new - pot
//   out_dev = [ |f|^2, |pot_new|^2, sum rho*(hpot+hpot0), sum rho*vxc ]
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_scf_update(const double* __restrict__ ppot, const double* __restrict__ vxc, const double* __restrict__ hpot,
             const double* __restrict__ hpot0, const double* __restrict__ rho, const double* __restrict__ pot,
             double* __restrict__ pot_new, double* __restrict__ f, long n, double* __restrict__ partial) {
  __shared__ double sh[8];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double pn = ppot[i] + 0.5 * vxc[i] + hpot[i] + hpot0[i];
    const double d = pn - pot[i];
    pot_new[i] = pn;
    if (f) f[i] = d;
    s0 += d * d;
    s1 += pn * pn;
    s2 += rho[i] * (hpot[i] + hpot0[i]);
    s3 += rho[i] * vxc[i];
  }
  double v[4] = {s0, s1, s2, s3};
  for (int q = 0; q < 4; ++q) {
    const double t = psc_block_sum<double, 256>(v[q], sh);
    if (threadIdx.x == 0) partial[(long)q * PSC_RED_BLOCKS + blockIdx.x] = t;
  }
}

__global__ void k_sum_slots(const double* partial, int nslots, double* out) {
  __shared__ double sh[8];
  for (int q = 0; q < nslots; ++q) {
    double s = 0.0;
    for (int i = threadIdx.x; i < PSC_RED_BLOCKS; i += 256) s += partial[(long)q * PSC_RED_BLOCKS + i];
    s = psc_block_sum<double, 256>(s, sh);
    if (threadIdx.x == 0) out[q] = s;
  }
}

extern "C" int psc_scf_update(psc_ctx* ctx, const double* ppot, const double* vxc, const double* hpot,
                              const double* hpot0, const double* rho, const double* pot, double* pot_new, double* f,
                              double* out_dev, void* stream) {
  if (!ctx) return 2;
  cudaStream_t st = (cudaStream_t)stream;
  k_scf_update<<<PSC_RED_BLOCKS, 256, 0, st>>>(ppot, vxc, hpot, hpot0, rho, pot, pot_new, f, ctx->n, ctx->red_partial);
  PSC_LAUNCH_CHECK(ctx);
  k_sum_slots<<<1, 256, 0, st>>>(ctx->red_partial, 4, out_dev);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}
