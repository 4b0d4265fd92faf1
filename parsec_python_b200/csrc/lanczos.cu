// Lanczos with a kept basis and the pieces that turn it into a starting
// subspace: the reference's Eigensolvers/lanczosForChsubsp.py (diagmeth 2,
// called by chsubsp.py) and Eigensolvers/lanczos.py (diagmeth 0/1).
//
//   psc_lanczos_run          m steps of the three-term recurrence without
//                            reorthogonalisation; the basis vectors are the
//                            columns of VV, alpha/beta stay on the device
//   psc_tridiag_eig          all eigenvalues of the Lanczos tridiagonal by
//                            Sturm-count multisection (one warp per value),
//                            eigenvectors of the lowest ones by inverse
//                            iteration (one warp per cluster of close values)
//   psc_orthonormalize_rank  CholeskyQR that drops numerically dependent
//                            columns first: W = VV X has near-copies of the
//                            same Ritz vector wherever the Lanczos tridiagonal
//                            has "ghost" eigenvalues
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

// ---------------------------------------------------------------------------
// Lanczos steps.  Each step is H v_j (the stencil + projector kernels) into
// VV[:, j+1], then three streaming passes with deterministic block sums:
//   1. f -= beta_{j-1} v_{j-1};   partial dots v_j . f
//   2. alpha_j = sum;  f -= alpha_j v_j;   partial sums f . f
//   3. beta_j = sqrt(sum);  v_{j+1} = f * (1 / beta_j)
// Every CTA of passes 2 and 3 adds the LZ_BLOCKS partials itself in a fixed
// order, so no separate reduction launch is needed and the result does not
// depend on scheduling.
// ---------------------------------------------------------------------------
constexpr int LZ_BLOCKS = 296;  // two CTAs per SM; also the number of partial sums
constexpr int LZ_NT = 256;

__device__ __forceinline__ double lz_partials(const double* __restrict__ part, double* sh, double* bc) {
  double s = 0.0;
  for (int i = threadIdx.x; i < LZ_BLOCKS; i += LZ_NT) s += part[i];
  s = psc_block_sum<double, LZ_NT>(s, sh);
  if (threadIdx.x == 0) *bc = s;
  __syncthreads();
  return *bc;
}

__global__ void __launch_bounds__(LZ_NT)
k_lz_sumsq(const double* __restrict__ x, long n, double* __restrict__ part) {
  __shared__ double sh[LZ_NT / 32];
  double s = 0.0;
  for (long i = blockIdx.x * (long)LZ_NT + threadIdx.x; i < n; i += (long)LZ_BLOCKS * LZ_NT) s += x[i] * x[i];
  s = psc_block_sum<double, LZ_NT>(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// v = x / ||x||  (lanczosForChsubsp.py:35, lanczos.py:40)
__global__ void __launch_bounds__(LZ_NT)
k_lz_normalize(const double* x, double* v, long n, const double* __restrict__ part) {  // x may be v
  __shared__ double sh[LZ_NT / 32];
  __shared__ double bc;
  const double nrm = sqrt(lz_partials(part, sh, &bc));
  for (long i = blockIdx.x * (long)LZ_NT + threadIdx.x; i < n; i += (long)LZ_BLOCKS * LZ_NT) v[i] = x[i] / nrm;
}

__global__ void __launch_bounds__(LZ_NT)
k_lz_pass1(const double* __restrict__ vj, const double* __restrict__ vjm1, const double* __restrict__ ab, int j,
           double* __restrict__ f, long n, double* __restrict__ part) {
  __shared__ double sh[LZ_NT / 32];
  const double bet = j > 0 ? ab[2 * (j - 1) + 1] : 0.0;
  double s = 0.0;
  for (long i = blockIdx.x * (long)LZ_NT + threadIdx.x; i < n; i += (long)LZ_BLOCKS * LZ_NT) {
    double w = f[i];
    if (j > 0) w = w - bet * vjm1[i];
    f[i] = w;
    s += vj[i] * w;
  }
  s = psc_block_sum<double, LZ_NT>(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(LZ_NT)
k_lz_pass2(const double* __restrict__ vj, double* __restrict__ f, long n, const double* __restrict__ part1,
           double* __restrict__ part2, double* __restrict__ ab, int j) {
  __shared__ double sh[LZ_NT / 32];
  __shared__ double bc;
  const double alp = lz_partials(part1, sh, &bc);
  double s = 0.0;
  for (long i = blockIdx.x * (long)LZ_NT + threadIdx.x; i < n; i += (long)LZ_BLOCKS * LZ_NT) {
    const double w = f[i] - alp * vj[i];
    f[i] = w;
    s += w * w;
  }
  s = psc_block_sum<double, LZ_NT>(s, sh);
  if (threadIdx.x == 0) {
    part2[blockIdx.x] = s;
    if (blockIdx.x == 0) ab[2 * j] = alp;
  }
}

__global__ void __launch_bounds__(LZ_NT)
k_lz_pass3(double* __restrict__ f, long n, const double* __restrict__ part2, double* __restrict__ ab, int j) {
  __shared__ double sh[LZ_NT / 32];
  __shared__ double bc;
  const double bet = sqrt(lz_partials(part2, sh, &bc));
  const double inv = 1.0 / bet;
  for (long i = blockIdx.x * (long)LZ_NT + threadIdx.x; i < n; i += (long)LZ_BLOCKS * LZ_NT) f[i] = f[i] * inv;
  if (blockIdx.x == 0 && threadIdx.x == 0) ab[2 * j + 1] = bet;
}

extern "C" int psc_lanczos_run(psc_ctx* ctx, const double* v_start, unsigned long long seed, int k0, int k1,
                               double* VV, long ldv, double* ab, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, VV && ab && ldv >= ctx->n, "lanczos_run: bad arguments");
  PSC_REQUIRE(ctx, k0 >= 0 && k1 >= k0, "lanczos_run: bad step range");
  cudaStream_t st = (cudaStream_t)stream;
  const long n = ctx->n;
  double* part1 = ctx->red_partial;
  double* part2 = ctx->red_partial + PSC_RED_BLOCKS;
  if (k0 == 0) {
    const double* x = v_start;
    if (!x) {
      // np.random.randn(n) (chsubsp.py:34, rsdft_solver.py:63-68)
      int rc = psc_random_impl(ctx, PSC_F64, 1, seed, VV, ldv, n, 1, st);
      if (rc) return rc;
      x = VV;
    }
    k_lz_sumsq<<<LZ_BLOCKS, LZ_NT, 0, st>>>(x, n, part1);
    PSC_LAUNCH_CHECK(ctx);
    k_lz_normalize<<<LZ_BLOCKS, LZ_NT, 0, st>>>(x, VV, n, part1);
    PSC_LAUNCH_CHECK(ctx);
  }
  for (int j = k0; j < k1; ++j) {
    const double* vj = VV + (long)j * ldv;
    const double* vjm1 = j > 0 ? VV + (long)(j - 1) * ldv : nullptr;
    double* f = VV + (long)(j + 1) * ldv;
    int rc = psc_apply_h_impl(ctx, PSC_F64, vj, ldv, f, ldv, nullptr, 0, 1, nullptr, 1.0, 0.0, 0.0, st);
    if (rc) return rc;
    k_lz_pass1<<<LZ_BLOCKS, LZ_NT, 0, st>>>(vj, vjm1, ab, j, f, n, part1);
    PSC_LAUNCH_CHECK(ctx);
    k_lz_pass2<<<LZ_BLOCKS, LZ_NT, 0, st>>>(vj, f, n, part1, part2, ab, j);
    PSC_LAUNCH_CHECK(ctx);
    k_lz_pass3<<<LZ_BLOCKS, LZ_NT, 0, st>>>(f, n, part2, ab, j);
    PSC_LAUNCH_CHECK(ctx);
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Symmetric tridiagonal eigensolver.  T has diagonal a_i = ab[2i] and
// off-diagonal e_i = ab[2i+1] (i < k-1), the layout psc_lanczos_run writes.
//
// Eigenvalues: the Sturm count c(x) (negative pivots of the LDL^T factors of
// T - x I) is the number of eigenvalues below x.  One warp finds eigenvalue i
// by multisection of the Gershgorin interval: each of its 32 lanes evaluates
// c at P = PSC_TRI_POINTS interior points (32 P in all, the P recurrences of
// a lane interleaved so that their divisions overlap), a ballot keeps the
// sub-interval with c(lo) <= i < c(hi), so every round gains log2(32 P + 1)
// bits (at most 16 rounds).
//
// Eigenvectors: inverse iteration, (T - lambda I) x_new = x, three times from
// a pseudo-random start, with Gaussian elimination with partial pivoting of
// the tridiagonal (a second superdiagonal appears where rows are
// interchanged) and pivots below eps |T| replaced by +-eps |T|.  Eigenvalues
// closer than crel |T| form a cluster handled by one warp in ascending order
// (crel = 1e-7 for the Lanczos tridiagonals; 1e-3, the reorthogonalisation
// gap of LAPACK's dstein, when the vectors must be orthonormal to ~1e-13):
// each later member's shift is moved at least 10 eps |T| above the previous
// one and its iterate is orthogonalised against the members before it after
// every solve (modified Gram-Schmidt).  The entry of largest magnitude of
// each eigenvector is made positive.
// ---------------------------------------------------------------------------
constexpr int TRI_MAX_K = 4096;

__device__ __forceinline__ void tri_load(const double* __restrict__ ab, int k, double* a, double* e, double* s_lo,
                                         double* s_hi, double* red) {
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    a[i] = ab[2 * i];
    e[i] = i + 1 < k ? ab[2 * i + 1] : 0.0;
  }
  __syncthreads();
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    const double r = fabs(e[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0);
    lo = fmin(lo, a[i] - r);
    hi = fmax(hi, a[i] + r);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if ((threadIdx.x & 31) == 0) { red[w] = lo; red[32 + w] = hi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < nw; ++q) { lo = fmin(lo, red[q]); hi = fmax(hi, red[32 + q]); }
    *s_lo = lo;
    *s_hi = hi;
  }
  __syncthreads();
}

#ifndef PSC_TRI_POINTS
#define PSC_TRI_POINTS 1   // Sturm counts per lane and multisection round (2 and 4 measured slower)
#endif

// Sturm counts at P points, the P recurrences interleaved so that their
// divisions overlap
template <int P>
__device__ __forceinline__ void sturm_counts(const double* a, const double* e, int k, const double (&x)[P],
                                             double pivmin, int (&c)[P]) {
  double q[P];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    q[p] = a[0] - x[p];
    if (fabs(q[p]) < pivmin) q[p] = -pivmin;
    c[p] = q[p] < 0.0;
  }
  for (int i = 1; i < k; ++i) {
    const double ai = a[i], e2 = e[i - 1] * e[i - 1];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      q[p] = (ai - x[p]) - e2 / q[p];
      if (fabs(q[p]) < pivmin) q[p] = -pivmin;
      c[p] += q[p] < 0.0;
    }
  }
}

template <int NT, int P>
__global__ void __launch_bounds__(NT) k_tri_bisect(const double* __restrict__ ab, int k, double* __restrict__ evals) {
  extern __shared__ double tri_sm[];
  __shared__ double red[64];
  __shared__ double s_lo, s_hi;
  double* a = tri_sm;
  double* e = tri_sm + k;
  tri_load(ab, k, a, e, &s_lo, &s_hi, red);
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (NT / 32) + (threadIdx.x >> 5);
  if (i >= k) return;
  const double tnorm = fmax(fabs(s_lo), fabs(s_hi));
  const double pivmin = DBL_MIN * fmax(1.0, tnorm * tnorm);
  const double pad = 4.0 * DBL_EPSILON * tnorm * k + 4.0 * pivmin;
  const double step = 1.0 / (32.0 * P + 1.0);
  double lo = s_lo - pad, hi = s_hi + pad;
  for (int round = 0; round < 16; ++round) {
    if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + pivmin) break;
    // point t = lane P + p of 32 P interior points; counts rise with t
    double x[P];
    int c[P];
#pragma unroll
    for (int p = 0; p < P; ++p) x[p] = lo + (hi - lo) * ((double)(lane * P + p + 1) * step);
    sturm_counts<P>(a, e, k, x, pivmin, c);
    int pf = P;   // this lane's first point with more than i eigenvalues below it
    double xhi = 0.0, xlo = 0.0;
#pragma unroll
    for (int p = P - 1; p >= 0; --p)
      if (c[p] > i) {
        pf = p;
        xhi = x[p];
        xlo = p > 0 ? x[p - 1] : 0.0;
      }
    const unsigned m = __ballot_sync(0xffffffffu, pf < P);
    const double xlast = x[P - 1];
    if (m == 0) {
      lo = __shfl_sync(0xffffffffu, xlast, 31);
    } else {
      const int f = __ffs(m) - 1;
      const int pff = __shfl_sync(0xffffffffu, pf, f);
      const double h = __shfl_sync(0xffffffffu, xhi, f);
      const double l_in = __shfl_sync(0xffffffffu, xlo, f);
      const double l_prev = __shfl_sync(0xffffffffu, xlast, f > 0 ? f - 1 : 0);
      hi = h;
      if (pff > 0) lo = l_in;
      else if (f > 0) lo = l_prev;
    }
  }
  if (lane == 0) evals[i] = 0.5 * (lo + hi);
}

__device__ __forceinline__ double tri_hash_unit(unsigned long long j, unsigned long long i) {
  unsigned long long z = (j * 0x9E3779B97F4A7C15ull) ^ (i + 0x632BE59BD9B4E019ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;  // [-1, 1)
}

__device__ __forceinline__ double warp_dot_col(const double* x, const double* y, int k, int lane) {
  double s = 0.0;
  for (int i = lane; i < k; i += 32) s += x[i] * y[i];
  return psc_warp_sum(s);
}

// LU with partial pivoting of T - lam I (one thread; sequential by nature):
// rd = inverted diagonal of U, du / du2 its two superdiagonals, dl the
// multipliers, piv 1 where rows i and i+1 were interchanged
__device__ __forceinline__ void tri_lu(const double* __restrict__ a, const double* __restrict__ e, int k, double lam,
                                       double tiny, double* __restrict__ rd, double* __restrict__ du,
                                       double* __restrict__ du2, double* __restrict__ dl, double* __restrict__ piv) {
  double dc = a[0] - lam;
  double uc = k > 1 ? e[0] : 0.0;
  for (int i = 0; i + 1 < k; ++i) {
    const double sub = e[i];
    const double dn = a[i + 1] - lam;
    const double un = i + 2 < k ? e[i + 1] : 0.0;
    if (fabs(dc) >= fabs(sub)) {
      const double d = fabs(dc) < tiny ? (dc < 0.0 ? -tiny : tiny) : dc;
      const double r = 1.0 / d;
      const double m = sub * r;
      rd[i] = r; du[i] = uc; du2[i] = 0.0; dl[i] = m; piv[i] = 0.0;
      dc = dn - m * uc;
      uc = un;
    } else {
      const double r = 1.0 / sub;
      const double m = dc * r;
      rd[i] = r; du[i] = dn; du2[i] = un; dl[i] = m; piv[i] = 1.0;
      dc = uc - m * dn;
      uc = -m * un;
    }
  }
  const double d = fabs(dc) < tiny ? (dc < 0.0 ? -tiny : tiny) : dc;
  rd[k - 1] = 1.0 / d;
}

// x <- (T - lam I)^{-1} x from the factors of tri_lu (one thread)
__device__ __forceinline__ void tri_lu_solve(double* __restrict__ x, int k, const double* __restrict__ rd,
                                             const double* __restrict__ du, const double* __restrict__ du2,
                                             const double* __restrict__ dl, const double* __restrict__ piv) {
  // forward: apply the row interchanges and multipliers
  double xi = x[0];
  for (int i = 0; i + 1 < k; ++i) {
    const double xn = x[i + 1];
    if (piv[i] == 0.0) {
      x[i] = xi;
      xi = xn - dl[i] * xi;
    } else {
      x[i] = xn;
      xi = xi - dl[i] * xn;
    }
  }
  x[k - 1] = xi;
  // backward with U (diagonal stored inverted)
  double x1 = x[k - 1] * rd[k - 1], x2 = 0.0;
  x[k - 1] = x1;
  for (int i = k - 2; i >= 0; --i) {
    const double v = (x[i] - du[i] * x1 - du2[i] * x2) * rd[i];
    x[i] = v;
    x2 = x1;
    x1 = v;
  }
}

// Eigenvectors of the tridiagonal T by inverse iteration, one warp per
// cluster of close eigenvalues (the members are orthogonalised against the
// earlier ones).  With one warp per CTA (NT = 32) the LU factors and the
// iterate live in shared memory (8k doubles with T); with NT = 128 the
// factors go to `work` (5k doubles per cluster start) and the iterate to Z.
template <int NT>
__global__ void __launch_bounds__(NT)
k_tri_invit(const double* __restrict__ ab, int k, const double* __restrict__ evals, int nvec, double* __restrict__ Z,
            long ldz, double crel, double* __restrict__ work) {
  constexpr bool SMEM = NT == 32;
  extern __shared__ double tri_sm[];
  __shared__ double red[64];
  __shared__ double s_lo, s_hi;
  double* a = tri_sm;
  double* e = tri_sm + k;
  tri_load(ab, k, a, e, &s_lo, &s_hi, red);
  const int lane = threadIdx.x & 31;
  const int s0 = blockIdx.x * (NT / 32) + (threadIdx.x >> 5);
  if (s0 >= nvec) return;
  // the floor keeps 1 / tiny and the squared iterates finite when T = 0
  const double tnorm = fmax(fmax(fabs(s_lo), fabs(s_hi)), 1e-100);
  const double ctol = crel * tnorm;
  if (s0 > 0 && evals[s0] - evals[s0 - 1] <= ctol) return;  // not the first of its cluster
  int s1 = s0 + 1;
  while (s1 < nvec && evals[s1] - evals[s1 - 1] <= ctol) ++s1;
  const double tiny = fmax(DBL_EPSILON * tnorm, DBL_MIN);
  const double pertol = 10.0 * DBL_EPSILON * tnorm;
  double* rd = SMEM ? tri_sm + 2 * k : work + (long)s0 * 5 * k;
  double* du = rd + k;
  double* du2 = du + k;
  double* dl = du2 + k;
  double* piv = dl + k;
  double lam_prev = 0.0;
  for (int j = s0; j < s1; ++j) {
    double lam = evals[j];
    if (j > s0) lam = fmax(lam, lam_prev + pertol);
    lam_prev = lam;
    double* z = Z + (long)j * ldz;
    double* x = SMEM ? piv + k : z;
    if (lane == 0) tri_lu(a, e, k, lam, tiny, rd, du, du2, dl, piv);
    for (int i = lane; i < k; i += 32) x[i] = tri_hash_unit(j, i);
    __syncwarp();
    for (int it = 0; it < 3; ++it) {
      const double nrm = sqrt(warp_dot_col(x, x, k, lane));
      const double sc = nrm > 0.0 ? 1.0 / nrm : 1.0;
      for (int i = lane; i < k; i += 32) x[i] *= sc;
      __syncwarp();
      if (lane == 0) tri_lu_solve(x, k, rd, du, du2, dl, piv);
      __syncwarp();
      for (int p = s0; p < j; ++p) {
        const double* zp = Z + (long)p * ldz;
        const double c = warp_dot_col(x, zp, k, lane);
        for (int i = lane; i < k; i += 32) x[i] -= c * zp[i];
        __syncwarp();
      }
    }
    // unit norm, largest entry positive
    const double nrm = sqrt(warp_dot_col(x, x, k, lane));
    double best = 0.0;
    for (int i = lane; i < k; i += 32)
      if (fabs(x[i]) > fabs(best)) best = x[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_xor_sync(0xffffffffu, best, o);
      if (fabs(other) > fabs(best) || (fabs(other) == fabs(best) && other > best)) best = other;
    }
    const double sc = (best < 0.0 ? -1.0 : 1.0) / nrm;
    for (int i = lane; i < k; i += 32) z[i] = x[i] * sc;
    __syncwarp();
  }
}

static int tri_smem(psc_ctx* ctx, const void* func, size_t bytes) {
  if (bytes > 48 * 1024) PSC_CUDA(ctx, cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return 0;
}

int psc_tridiag_eig_impl(psc_ctx* ctx, const double* ab, int k, int nvec, double* evals, double* Z, long ldz,
                         double crel, cudaStream_t st) {
  PSC_REQUIRE(ctx, ab && evals && k >= 1 && k <= TRI_MAX_K, "tridiag_eig: k out of range");
  PSC_REQUIRE(ctx, nvec >= 0 && nvec <= k && (nvec == 0 || (Z && ldz >= k)), "tridiag_eig: bad eigenvector block");
  const size_t smem = 2 * (size_t)k * sizeof(double);
  // up to k = 512 one warp per CTA, so that the latency-bound warps get an SM
  // scheduler each; beyond, eight warps share each copy of T in shared memory
  const bool solo = k <= 512;
  if (solo) {
    if (tri_smem(ctx, (const void*)k_tri_bisect<32, PSC_TRI_POINTS>, smem)) return 1;
    k_tri_bisect<32, PSC_TRI_POINTS><<<k, 32, smem, st>>>(ab, k, evals);
  } else {
    if (tri_smem(ctx, (const void*)k_tri_bisect<256, PSC_TRI_POINTS>, smem)) return 1;
    k_tri_bisect<256, PSC_TRI_POINTS><<<psc_div_up(k, 8), 256, smem, st>>>(ab, k, evals);
  }
  PSC_LAUNCH_CHECK(ctx);
  if (nvec == 0) return 0;
  const size_t need = 5 * (size_t)k * nvec;
  if (need > ctx->tri_work_doubles) {
    psc_dfree(ctx->tri_work);
    ctx->tri_work = nullptr;
    ctx->tri_work_doubles = 0;
    PSC_CUDA(ctx, psc_dmalloc(&ctx->tri_work, need * sizeof(double)));
    ctx->tri_work_doubles = need;
  }
  if (solo) {
    const size_t smem_iv = 8 * (size_t)k * sizeof(double);   // T, the LU factors and the iterate
    if (tri_smem(ctx, (const void*)k_tri_invit<32>, smem_iv)) return 1;
    k_tri_invit<32><<<nvec, 32, smem_iv, st>>>(ab, k, evals, nvec, Z, ldz, crel, ctx->tri_work);
  } else {
    if (tri_smem(ctx, (const void*)k_tri_invit<128>, smem)) return 1;
    k_tri_invit<128><<<psc_div_up(nvec, 4), 128, smem, st>>>(ab, k, evals, nvec, Z, ldz, crel, ctx->tri_work);
  }
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

extern "C" int psc_tridiag_eig(psc_ctx* ctx, const double* ab, int k, int nvec, double* evals, double* Z, long ldz,
                               void* stream) {
  if (!ctx) return 2;
  return psc_tridiag_eig_impl(ctx, ab, k, nvec, evals, Z, ldz, 1e-7, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Rank-revealing orthonormalisation.  S = W^T W; a Cholesky sweep in column
// order keeps column j when the squared norm of its component orthogonal to
// the kept columns before it exceeds tol * |w_j|^2 and drops it otherwise
// (dropped rows take no part in later updates).  The kept columns are
// gathered into T and orthonormalised by CholeskyQR2.  With tol = 1e-10 a
// kept column has a relative residual above 1e-5, so the kept block has a
// condition number far inside CholeskyQR2's FP64 range.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_cholesky_drop(double* A, int k, double tol, int* keep) {
  __shared__ double d0[PSC_MAX_K];
  __shared__ int kept;
  for (int i = threadIdx.x; i < k; i += blockDim.x) d0[i] = A[i + (long)i * k];
  for (int j = 0; j < k; ++j) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const double d = A[j + (long)j * k];
      const int ok = d0[j] > 0.0 && d > tol * d0[j];
      keep[j] = ok;
      kept = ok;
      if (ok) A[j + (long)j * k] = sqrt(d);
    }
    __syncthreads();
    if (!kept) continue;
    const double rjj = A[j + (long)j * k];
    for (int c = j + 1 + threadIdx.x; c < k; c += blockDim.x) A[j + (long)c * k] /= rjj;
    __syncthreads();
    const int m = k - j - 1;
    for (long e = threadIdx.x; e < (long)m * m; e += blockDim.x) {
      const int r = j + 1 + (int)(e % m), c = j + 1 + (int)(e / m);
      if (r <= c) A[r + (long)c * k] -= A[j + (long)r * k] * A[j + (long)c * k];
    }
  }
}

template <typename T>
__global__ void k_gather_cols(const T* __restrict__ W, long ld, const int* __restrict__ idx, int r, long n,
                              T* __restrict__ O) {
  for (int c = blockIdx.y; c < r; c += gridDim.y) {
    const T* src = W + (long)idx[c] * ld;
    T* dst = O + (long)c * ld;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) dst[i] = src[i];
  }
}

extern "C" int psc_orthonormalize_rank(psc_ctx* ctx, int dtype, void* W, void* T, long ld, int k, double tol,
                                       int* rank, int* which, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, W && T && W != T && ld >= ctx->n && rank && which, "orthonormalize_rank: bad arguments");
  PSC_REQUIRE(ctx, tol > 0.0 && tol < 1.0, "orthonormalize_rank: tol must be in (0, 1)");
  cudaStream_t st = (cudaStream_t)stream;
  if (psc_ensure_dense(ctx, k)) return 1;
  int rc = psc_gram_impl(ctx, dtype, W, ld, W, ld, k, ctx->gram, 2, st);
  if (rc) return rc;
  int* keep_dev = reinterpret_cast<int*>(ctx->tri);  // k ints in the k x k scratch
  k_cholesky_drop<<<1, 1024, 0, st>>>(ctx->gram, k, tol, keep_dev);
  PSC_LAUNCH_CHECK(ctx);
  std::vector<int> keep(k);
  PSC_CUDA(ctx, cudaMemcpyAsync(keep.data(), keep_dev, k * sizeof(int), cudaMemcpyDeviceToHost, st));
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  std::vector<int> idx;
  for (int j = 0; j < k; ++j)
    if (keep[j]) idx.push_back(j);
  const int r = (int)idx.size();
  *rank = r;
  *which = 0;
  if (r == 0) return 0;
  PSC_CUDA(ctx, cudaMemcpyAsync(keep_dev, idx.data(), r * sizeof(int), cudaMemcpyHostToDevice, st));
  dim3 grid(psc_div_up(ctx->n, 256 * 8), std::min(r, 1024));
  if (dtype == PSC_F64)
    k_gather_cols<double><<<grid, 256, 0, st>>>((const double*)W, ld, keep_dev, r, ctx->n, (double*)T);
  else
    k_gather_cols<float><<<grid, 256, 0, st>>>((const float*)W, ld, keep_dev, r, ctx->n, (float*)T);
  PSC_LAUNCH_CHECK(ctx);
  // the host copy of idx must outlive the upload above
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  int w2 = 0;
  rc = psc_orthonormalize(ctx, dtype, T, W, ld, r, 2, &w2, st);
  if (rc) return rc;
  *which = w2 == 0 ? 1 : 0;
  return 0;
}

// ---------------------------------------------------------------------------
// The chefsi1 spectrum bound (Eigensolvers/lanczosForChefsi1.py:5-99 with
// m = 6): six steps of the recurrence above from a standard normal start,
// then bound = max |theta| + beta_6 over the eigenvalues theta of T_6.
// ---------------------------------------------------------------------------
__global__ void k_lz_bound6(const double* __restrict__ ev, const double* __restrict__ ab, int m, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double mx = 0.0;
    for (int i = 0; i < m; ++i) mx = fmax(mx, fabs(ev[i]));
    out[0] = mx + ab[2 * (m - 1) + 1];
  }
}

int psc_lanczos_bound_basis(psc_ctx* ctx, unsigned long long seed, const double* v_start, double* out_dev,
                            cudaStream_t st) {
  constexpr int m = 6;
  const long n = ctx->n;
  if (!ctx->lz_basis) PSC_CUDA(ctx, psc_dmalloc(&ctx->lz_basis, (size_t)(m + 1) * n * sizeof(double)));
  double* ab = ctx->scalars + 160;  // [2m] alpha, beta
  double* ev = ctx->scalars + 176;  // [m]
  int rc = psc_lanczos_run(ctx, v_start, seed, 0, m, ctx->lz_basis, n, ab, st);
  if (rc) return rc;
  rc = psc_tridiag_eig(ctx, ab, m, 0, ev, nullptr, 0, st);
  if (rc) return rc;
  k_lz_bound6<<<1, 32, 0, st>>>(ev, ab, m, out_dev);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}
