// Context lifetime, error reporting, species spline tables, deterministic
// reductions and the counter-based random generator.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <cmath>
#include <cstring>
#include <mutex>

static std::string g_last_error;
static std::mutex g_err_mu;

void psc_set_error(psc_ctx* ctx, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_last_error = msg;
}

extern "C" const char* psc_last_error(const psc_ctx* ctx) {
  if (ctx) return ctx->last_error.c_str();
  return g_last_error.c_str();
}

extern "C" int psc_version(void) { return PSC_ABI_VERSION; }

// Finite-difference weights of -h^2 d2/dx2 summed over the axes
// (Laplacian/fd3d.py:49-94): orders <=2, <=4, <=6, else 8.
static void fd_weights(int order, double* c0, double* c, int* radius) {
  for (int i = 0; i < 4; ++i) c[i] = 0.0;
  if (order <= 2) {
    *c0 = 6.0; c[0] = -1.0; *radius = 1;
  } else if (order <= 4) {
    *c0 = 15.0 / 2.0; c[0] = -4.0 / 3.0; c[1] = 1.0 / 12.0; *radius = 2;
  } else if (order <= 6) {
    *c0 = 49.0 / 6.0; c[0] = -3.0 / 2.0; c[1] = 3.0 / 20.0; c[2] = -1.0 / 90.0; *radius = 3;
  } else {
    *c0 = 205.0 / 24.0; c[0] = -8.0 / 5.0; c[1] = 1.0 / 5.0; c[2] = -8.0 / 315.0; c[3] = 1.0 / 560.0;
    *radius = 4;
  }
}

extern "C" int psc_ctx_create(int nx, int ny, int nz, double h, int fd_order, psc_ctx** out) {
  if (!out) { psc_set_error(nullptr, "psc_ctx_create: out is NULL"); return 2; }
  *out = nullptr;
  if (nx < 1 || ny < 1 || nz < 1 || !(h > 0.0)) {
    psc_set_error(nullptr, "psc_ctx_create: grid dimensions must be >= 1 and h > 0");
    return 2;
  }
  long n = (long)nx * ny * nz;
  if (n > (long)INT32_MAX / 2) { psc_set_error(nullptr, "psc_ctx_create: grid too large"); return 2; }
  psc_ctx* ctx = new psc_ctx();
  cudaGetDevice(&ctx->device);
  ctx->nx = nx; ctx->ny = ny; ctx->nz = nz; ctx->n = n; ctx->h = h; ctx->fd_order = fd_order;
  double c0, c[4];
  fd_weights(fd_order, &c0, c, &ctx->radius);
  const double ih2 = 1.0 / (h * h);
  ctx->lap_c0 = c0 * ih2;
  ctx->ham_c0 = 0.5 * (c0 * ih2);
  for (int i = 0; i < 4; ++i) {
    ctx->lap_c[i] = c[i] * ih2;
    ctx->ham_c[i] = 0.5 * (c[i] * ih2);
  }
  {
    // the weights' FP32 rounding errors break the sum rule c0 + 6 sum_d c_d = 0
    double rs = (double)(float)ctx->ham_c0 - ctx->ham_c0;
    for (int i = 0; i < 4; ++i) rs += 6.0 * ((double)(float)ctx->ham_c[i] - ctx->ham_c[i]);
    ctx->sumrule32 = -rs;
  }
  ctx->species.resize(32);
  auto fail = [&](cudaError_t e, const char* what) {
    psc_set_error(nullptr, std::string("psc_ctx_create: ") + what + ": " + cudaGetErrorString(e));
    psc_ctx_destroy(ctx);
    return 1;
  };
  cudaError_t e;
  if ((e = psc_dmalloc(&ctx->pot64, n * sizeof(double))) != cudaSuccess) return fail(e, "pot64");
  if ((e = psc_dmalloc(&ctx->pot32, n * sizeof(float))) != cudaSuccess) return fail(e, "pot32");
  if ((e = cudaMemset(ctx->pot64, 0, n * sizeof(double))) != cudaSuccess) return fail(e, "pot64");
  if ((e = cudaMemset(ctx->pot32, 0, n * sizeof(float))) != cudaSuccess) return fail(e, "pot32");
  if ((e = psc_dmalloc(&ctx->cheb_coef, (PSC_MAX_DEG + 1) * 3 * sizeof(double))) != cudaSuccess)
    return fail(e, "coef");
  if ((e = psc_dmalloc(&ctx->red_partial, (size_t)PSC_RED_SLOTS * PSC_RED_BLOCKS * sizeof(double))) !=
      cudaSuccess)
    return fail(e, "partials");
  if ((e = psc_dmalloc(&ctx->scalars, 256 * sizeof(double))) != cudaSuccess) return fail(e, "scalars");
  if ((e = cudaMemset(ctx->scalars, 0, 256 * sizeof(double))) != cudaSuccess) return fail(e, "scalars");
  if ((e = cudaMallocHost(&ctx->host_scalars, 256 * sizeof(double))) != cudaSuccess)
    return fail(e, "host scalars");
  if ((e = psc_dmalloc(&ctx->dev_status, 8 * sizeof(int))) != cudaSuccess) return fail(e, "status");
  if ((e = cudaMemset(ctx->dev_status, 0, 8 * sizeof(int))) != cudaSuccess) return fail(e, "status");
  if ((e = psc_dmalloc(&ctx->lz_v, 3 * n * sizeof(double))) != cudaSuccess) return fail(e, "lanczos");
  if ((e = psc_dmalloc(&ctx->cg_r, n * sizeof(double))) != cudaSuccess) return fail(e, "cg");
  if ((e = psc_dmalloc(&ctx->cg_p, n * sizeof(double))) != cudaSuccess) return fail(e, "cg");
  if ((e = psc_dmalloc(&ctx->cg_ap, n * sizeof(double))) != cudaSuccess) return fail(e, "cg");
  *out = ctx;
  return 0;
}

static void free_species(psc_species& s) {
  for (int i = 0; i < 5; ++i) {
    psc_dfree(s.x[i]); psc_dfree(s.z[i]); psc_dfree(s.c[i]); psc_dfree(s.d[i]);
    s.x[i] = s.z[i] = s.c[i] = s.d[i] = nullptr;
  }
  s.valid = 0;
}

void psc_free_projectors(psc_ctx* ctx);

extern "C" int psc_ctx_destroy(psc_ctx* ctx) {
  if (!ctx) return 0;
  for (auto& s : ctx->species) free_species(s);
  psc_free_projectors(ctx);
  psc_dfree(ctx->pot64); psc_dfree(ctx->pot32); psc_dfree(ctx->cheb_coef); psc_dfree(ctx->red_partial);
  psc_dfree(ctx->scalars); cudaFreeHost(ctx->host_scalars); psc_dfree(ctx->dev_status);
  psc_dfree(ctx->gram); psc_dfree(ctx->gram2); psc_dfree(ctx->evec); psc_dfree(ctx->tri);
  psc_dfree(ctx->gram_partial); psc_dfree(ctx->lz_v); psc_dfree(ctx->cg_r); psc_dfree(ctx->cg_p);
  psc_dfree(ctx->cg_ap); psc_dfree(ctx->cg_part); psc_dfree(ctx->mix_dx); psc_dfree(ctx->mix_df);
  psc_dfree(ctx->mix_nv); psc_dfree(ctx->mix_tmp); psc_dfree(ctx->mix_coef); psc_dfree(ctx->mix_partial);
  psc_dfree(ctx->cg_x); psc_dfree(ctx->eig_work); psc_dfree(ctx->cg_p2); psc_dfree(ctx->cg_ro); psc_dfree(ctx->cg_bar);
  psc_dfree(ctx->tc_part); psc_dfree(ctx->tc_pairs); psc_dfree(ctx->tri_work); psc_dfree(ctx->col_norm_part); psc_dfree(ctx->tsplit);
  for (auto& e : ctx->st_sched) psc_dfree(e.dev);
  psc_dfree(ctx->dm_pairs);
  psc_dfree(ctx->conv_wt);
  psc_dfree(ctx->pw_buf);
  psc_dfree(ctx->dens_w);
  for (int a = 0; a < 3; ++a) { psc_dfree(ctx->spec_S[a]); psc_dfree(ctx->spec_lam[a]); }
  psc_dfree(ctx->spec_tmp); psc_dfree(ctx->lz_basis);
  if (ctx->cg_exec) cudaGraphExecDestroy(ctx->cg_exec);
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  delete ctx;
  return 0;
}

extern "C" int psc_ctx_info(const psc_ctx* ctx, long* out /* [8] */) {
  if (!ctx || !out) return 2;
  out[0] = ctx->nx; out[1] = ctx->ny; out[2] = ctx->nz; out[3] = ctx->n;
  out[4] = ctx->nl_atoms; out[5] = ctx->nl_points; out[6] = ctx->nl_touched; out[7] = ctx->radius;
  return 0;
}

// ---------------------------------------------------------------------------
// species spline tables (host construction, V_ion/preProcess.py:4-26,
// Splines/fspline.py:5-45, Splines/trid.py:3-32)
// ---------------------------------------------------------------------------
static void prune_knots(const std::vector<double>& v, std::vector<int>& keep) {
  keep.clear();
  keep.push_back(0);
  const int n = (int)v.size();
  for (int i = 1; i < n - 1; ++i)
    if (std::fabs(v[i] - v[i - 1]) > 10e-6) keep.push_back(i);
  keep.push_back(n - 1);
}

static int natural_spline(const std::vector<double>& xi, const std::vector<double>& yi,
                          std::vector<double>& z, std::vector<double>& c, std::vector<double>& d) {
  const int np1 = (int)xi.size();
  const int n = np1 - 1;
  if (n < 2) return 1;
  std::vector<double> h(n), r(n);
  for (int i = 0; i < n; ++i) h[i] = xi[i + 1] - xi[i];
  for (int i = 0; i < n; ++i) r[i] = (yi[i + 1] - yi[i]) / h[i];
  const int m = n - 1;
  std::vector<double> rr(m), a(m), cu(m), dd(m);
  for (int i = 0; i < m; ++i) {
    rr[i] = r[i + 1] - r[i];
    a[i] = h[i];
    cu[i] = h[i + 1];
    dd[i] = 2 * (h[i] + h[i + 1]);
  }
  for (int k = 1; k < m; ++k) {
    double piv = a[k] / dd[k - 1];
    dd[k] = dd[k] - piv * cu[k - 1];
    rr[k] = rr[k] - piv * rr[k - 1];
  }
  rr[m - 1] = rr[m - 1] / dd[m - 1];
  for (int j = m - 2; j >= 0; --j) rr[j] = (rr[j] - cu[j] * rr[j + 1]) / dd[j];
  z.assign(np1, 0.0);
  for (int i = 0; i < m; ++i) z[i + 1] = rr[i];
  c.resize(n); d.resize(n);
  for (int i = 0; i < n; ++i) {
    c[i] = (yi[i] / h[i]) - (z[i] * h[i]);
    d[i] = (yi[i + 1] / h[i]) - (z[i + 1] * h[i]);
  }
  return 0;
}

extern "C" int psc_set_species(psc_ctx* ctx, int species_id, int nknots, const double* table,
                               double zvalue, double rcut) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, species_id >= 0 && species_id < (int)ctx->species.size(), "species id out of range");
  PSC_REQUIRE(ctx, table && nknots >= 4, "species table needs >= 4 knots");
  cudaSetDevice(ctx->device);
  psc_species& s = ctx->species[species_id];
  free_species(s);
  // table is row-major nknots x 7: radius, charge, hartree, pot_P, pot_S, wfn_P, wfn_S
  std::vector<double> r(nknots), cols[5];
  for (int i = 0; i < 5; ++i) cols[i].resize(nknots);
  for (int i = 0; i < nknots; ++i) {
    const double* row = table + 7 * (long)i;
    r[i] = row[0];
    cols[0][i] = row[1];
    cols[1][i] = row[2];
    cols[2][i] = row[4];
    cols[3][i] = row[5];
    cols[4][i] = row[3] - row[4];
  }
  for (int f = 0; f < 5; ++f) {
    std::vector<int> keep;
    prune_knots(cols[f], keep);
    std::vector<double> xk(keep.size()), yk(keep.size()), z, c, d;
    for (size_t i = 0; i < keep.size(); ++i) { xk[i] = r[keep[i]]; yk[i] = cols[f][keep[i]]; }
    PSC_REQUIRE(ctx, natural_spline(xk, yk, z, c, d) == 0, "spline needs >= 3 distinct knots");
    const int nk = (int)xk.size();
    s.nk[f] = nk;
    PSC_CUDA(ctx, psc_dmalloc(&s.x[f], nk * sizeof(double)));
    PSC_CUDA(ctx, psc_dmalloc(&s.z[f], nk * sizeof(double)));
    PSC_CUDA(ctx, psc_dmalloc(&s.c[f], (nk - 1) * sizeof(double)));
    PSC_CUDA(ctx, psc_dmalloc(&s.d[f], (nk - 1) * sizeof(double)));
    PSC_CUDA(ctx, cudaMemcpy(s.x[f], xk.data(), nk * sizeof(double), cudaMemcpyHostToDevice));
    PSC_CUDA(ctx, cudaMemcpy(s.z[f], z.data(), nk * sizeof(double), cudaMemcpyHostToDevice));
    PSC_CUDA(ctx, cudaMemcpy(s.c[f], c.data(), (nk - 1) * sizeof(double), cudaMemcpyHostToDevice));
    PSC_CUDA(ctx, cudaMemcpy(s.d[f], d.data(), (nk - 1) * sizeof(double), cudaMemcpyHostToDevice));
  }
  s.zvalue = zvalue;
  s.rcut = rcut;
  s.valid = 1;
  return 0;
}

// Export of the host spline construction so the tables can be checked
// against the reference's fspline/preProcess on the CPU.
extern "C" int psc_spline_coeffs(int nknots, const double* x, const double* y, int* nkeep,
                                 double* xk_out, double* z_out, double* c_out, double* d_out) {
  std::vector<double> yv(y, y + nknots), xk, yk, z, c, d;
  std::vector<int> keep;
  prune_knots(yv, keep);
  for (int i : keep) { xk.push_back(x[i]); yk.push_back(y[i]); }
  if (natural_spline(xk, yk, z, c, d)) { psc_set_error(nullptr, "spline needs >= 3 knots"); return 2; }
  *nkeep = (int)xk.size();
  if (xk_out) std::memcpy(xk_out, xk.data(), xk.size() * sizeof(double));
  if (z_out) std::memcpy(z_out, z.data(), z.size() * sizeof(double));
  if (c_out) std::memcpy(c_out, c.data(), c.size() * sizeof(double));
  if (d_out) std::memcpy(d_out, d.data(), d.size() * sizeof(double));
  return 0;
}

// ---------------------------------------------------------------------------
// deterministic multi-dot
// ---------------------------------------------------------------------------
struct dot_args {
  const double* a[PSC_RED_SLOTS];
  const double* b[PSC_RED_SLOTS];
};

template <int NT>
__global__ void __launch_bounds__(NT) k_dots_partial(dot_args args, int nslots, long n, double* partial) {
  __shared__ double sh[NT / 32];
  const long chunk = (n + gridDim.x - 1) / gridDim.x;
  const long lo = chunk * blockIdx.x;
  const long hi = min(n, lo + chunk);
  for (int s = 0; s < nslots; ++s) {
    const double* a = args.a[s];
    const double* b = args.b[s];
    double acc = 0.0;
    for (long i = lo + threadIdx.x; i < hi; i += NT) acc += a[i] * b[i];
    acc = psc_block_sum<double, NT>(acc, sh);
    if (threadIdx.x == 0) partial[(long)s * PSC_RED_BLOCKS + blockIdx.x] = acc;
  }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_dots_final(const double* partial, int nslots, double* out) {
  __shared__ double sh[NT / 32];
  for (int s = 0; s < nslots; ++s) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < PSC_RED_BLOCKS; i += NT) acc += partial[(long)s * PSC_RED_BLOCKS + i];
    acc = psc_block_sum<double, NT>(acc, sh);
    if (threadIdx.x == 0) out[s] = acc;
  }
}

int psc_dots(psc_ctx* ctx, int nslots, const double* const* a, const double* const* b, long n,
             double* out_dev, cudaStream_t st) {
  PSC_REQUIRE(ctx, nslots >= 1 && nslots <= PSC_RED_SLOTS, "psc_dots: bad slot count");
  dot_args args;
  for (int s = 0; s < nslots; ++s) { args.a[s] = a[s]; args.b[s] = b[s]; }
  k_dots_partial<256><<<PSC_RED_BLOCKS, 256, 0, st>>>(args, nslots, n, ctx->red_partial);
  PSC_LAUNCH_CHECK(ctx);
  k_dots_final<256><<<1, 256, 0, st>>>(ctx->red_partial, nslots, out_dev);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_dot(psc_ctx* ctx, const double* a, const double* b, long n, double* out_dev,
                       void* stream) {
  if (!ctx) return 2;
  return psc_dots(ctx, 1, &a, &b, n, out_dev, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// counter-based random numbers (SplitMix64 finaliser on (seed, index))
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double u01(uint64_t seed, uint64_t i) {
  // 53 random bits -> [0, 1)
  return (double)(mix64(seed * 0x632BE59BD9B4E019ull + i) >> 11) * (1.0 / 9007199254740992.0);
}

template <typename T>
__global__ void k_random(T* out, long ld, long rows, int cols, uint64_t seed, int dist) {
  const long total = rows * (long)cols;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const long r = t % rows, c = t / rows;
    double v;
    if (dist == 0) {
      v = u01(seed, 2 * (uint64_t)t);
    } else {  // Box-Muller normal
      double u1 = u01(seed, 2 * (uint64_t)t);
      double u2 = u01(seed, 2 * (uint64_t)t + 1);
      u1 = 1.0 - u1;  // (0, 1]
      v = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    }
    out[r + c * ld] = (T)v;
  }
}

int psc_random_impl(psc_ctx* ctx, int dtype, int dist, unsigned long long seed, void* out, long ld,
                    long rows, int cols, cudaStream_t st) {
  PSC_REQUIRE(ctx, ld >= rows && rows > 0 && cols > 0, "psc_random: bad shape");
  const int nb = 148 * 8;
  if (dtype == PSC_F64)
    k_random<double><<<nb, 256, 0, st>>>((double*)out, ld, rows, cols, seed, dist);
  else
    k_random<float><<<nb, 256, 0, st>>>((float*)out, ld, rows, cols, seed, dist);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_random(psc_ctx* ctx, int dtype, int dist, unsigned long long seed, void* out,
                          long ld, long rows, int cols, void* stream) {
  if (!ctx) return 2;
  return psc_random_impl(ctx, dtype, dist, seed, out, ld, rows, cols, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// small utilities
// ---------------------------------------------------------------------------
__global__ void k_cast_d2f(const double* a, float* b, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
__global__ void k_cast_f2d(const float* a, double* b, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    b[i] = (double)a[i];
}

extern "C" int psc_cast(psc_ctx* ctx, int to_dtype, const void* src, void* dst, long n, void* stream) {
  if (!ctx) return 2;
  cudaStream_t st = (cudaStream_t)stream;
  if (to_dtype == PSC_F32)
    k_cast_d2f<<<148 * 8, 256, 0, st>>>((const double*)src, (float*)dst, n);
  else
    k_cast_f2d<<<148 * 8, 256, 0, st>>>((const float*)src, (double*)dst, n);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

__global__ void k_cast_d2f_shift(const double* a, float* b, long n, double shift) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    b[i] = (float)(a[i] + shift);
}

// pot32 = fl(pot64 + shift): with weights mode 2 the FP32 weights' sum-rule
// correction rides on the FP32 potential (the stencil's pot x term), so the
// FP32 kernel needs no term of its own.  Each point's rounding error is as
// random as fl(pot64)'s own, and the systematic shift survives it.
int psc_recast_pot32(psc_ctx* ctx, cudaStream_t st) {
  ctx->pot32_shift = ctx->stencil_comp == 2 ? ctx->sumrule32 : 0.0;
  k_cast_d2f_shift<<<148 * 8, 256, 0, st>>>(ctx->pot64, ctx->pot32, ctx->n, ctx->pot32_shift);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_set_potential(psc_ctx* ctx, const double* pot, void* stream) {
  if (!ctx || !pot) return 2;
  cudaStream_t st = (cudaStream_t)stream;
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->pot64, pot, ctx->n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  return psc_recast_pot32(ctx, st);
}

extern "C" int psc_status(psc_ctx* ctx, int* host_flags /* [8] */, int clear, void* stream) {
  if (!ctx) return 2;
  cudaStream_t st = (cudaStream_t)stream;
  PSC_CUDA(ctx, cudaMemcpyAsync(host_flags, ctx->dev_status, 8 * sizeof(int), cudaMemcpyDeviceToHost, st));
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  if (clear) PSC_CUDA(ctx, cudaMemsetAsync(ctx->dev_status, 0, 8 * sizeof(int), st));
  return 0;
}

// Polls of every bounded device-side wait (stencil bulk-copy pipeline,
// tensor-core Gram, block-product and convolution pipelines; the CG grid barrier waits 4x
// as long) before the CTA gives up and records its status word.  polls < 0
// restores the default.  A test can set 0 to make every wait run out at once
// and check that the failure is reported and the context stays usable.
extern "C" int psc_set_wait_limit(psc_ctx* ctx, long polls) {
  if (!ctx) return 2;
  ctx->wait_limit = polls < 0 ? PSC_WAIT_DEFAULT : polls;
  return 0;
}

// out = a*x + b*y (y may be NULL)
__global__ void k_axpby(const double* __restrict__ x, const double* __restrict__ y, double a, double b,
                        double* __restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = y ? a * x[i] + b * y[i] : a * x[i];
}

extern "C" int psc_axpby(psc_ctx* ctx, const double* x, const double* y, double a, double b, double* out, long n,
                         void* stream) {
  if (!ctx) return 2;
  k_axpby<<<148 * 8, 256, 0, (cudaStream_t)stream>>>(x, y, a, b, out, n);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

#include <atomic>
#include <mutex>
static std::atomic<long long> g_launches{0};

cudaError_t psc_dmalloc_bytes(void** p, size_t bytes) {
  static std::mutex mu;
  static bool pool_ready[64] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64) {
    std::lock_guard<std::mutex> lk(mu);
    if (!pool_ready[dev]) {
      cudaMemPool_t pool;
      e = cudaDeviceGetDefaultMemPool(&pool, dev);
      if (e != cudaSuccess) return e;
      uint64_t keep = ~0ull;
      e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) return e;
      pool_ready[dev] = true;
    }
  }
  e = cudaMallocAsync(p, bytes, cudaStreamLegacy);
  if (e != cudaSuccess) return e;
  // a block reused from the pool may still be the target of work queued
  // before its free; make it safe for any stream
  return cudaStreamSynchronize(cudaStreamLegacy);
}

void psc_dfree(void* p) {
  if (p) cudaFreeAsync(p, cudaStreamLegacy);
}
void psc_note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
extern "C" long long psc_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }
