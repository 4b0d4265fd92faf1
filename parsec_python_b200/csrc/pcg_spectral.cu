// Preconditioned Hartree solve (cg_prec = 1): conjugate gradients on
// A = -Lap_h with a spectral preconditioner, in the preconditioned form of
// Eigensolvers/pcg.py:7-85 (z = M r, p = z, ro = z.r, stop when
// z.r <= tol^2 z0.r0).
//
// The preconditioner.  On the nx x ny x nz box with zero values outside, the
// orthonormal discrete sine transform (DST-I) of each axis,
//   S[j][k] = sqrt(2 / (m + 1)) sin(pi (j + 1)(k + 1) / (m + 1)),
// diagonalises the same finite-difference stencil continued by odd
// reflection across the faces; its eigenvalues are the stencil's symbol,
//   Lambda = lap_c0 + sum_axes sum_d 2 lap_c[d] cos(d theta_axis),
//   theta = pi (k + 1) / (m + 1).
// For the 2nd-order stencil that operator is A itself; for wider stencils it
// differs from A only in the R planes next to each face (A reads zeros
// there, the reflected operator reads mirrored values), so
//   M = S_z S_y S_x Lambda^-1 S_x S_y S_z
// is a symmetric positive definite approximate inverse whose error is
// confined to the boundary layer.  S is symmetric and its own inverse.
//
// Each application is five passes over the grid, each a batch of small
// dense products of 16 grid lines by S held in shared memory: x forward, y
// forward, z forward + 1/Lambda + z back in one kernel, y back, x back.  The
// grid lines of a tile are loaded and stored in coalesced order (rows of x
// for the x axis, 16 consecutive points of every y row or z plane for the
// others).  FP64 throughout.
//
// The reference's own cg_prec = 1 path has nothing to reproduce: its CPU
// branch passes the string "precLU" where pcg.py calls a function
// (rsdft_solver.py:339 into pcg.py:43) and its GPU twin ignores the
// preconditioner (pcg_gpu.py:38-41).
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>
#include <cmath>
#include <vector>

constexpr int SP_W = 16;    // grid lines per tile
constexpr int SP_NT = 128;  // 8 groups of 2 lines x 16 groups of output modes
constexpr int SP_RPT = SP_W / 8;  // lines per thread
constexpr int SP_MAXM = 128;

// C[i][j] = sum_k T[i][k] S[k][j], i < w, j < m; thread (ig, jg) owns
// i = SP_RPT ig .. SP_RPT ig + SP_RPT - 1 and j = jg + 16 q
template <int QJ>
__device__ __forceinline__ void sp_tile_mm(const double* __restrict__ T, int tl, const double* __restrict__ S, int mp,
                                           int m, double acc[SP_RPT][QJ]) {
  const int ig = threadIdx.x >> 4, jg = threadIdx.x & 15;
#pragma unroll
  for (int a = 0; a < SP_RPT; ++a)
#pragma unroll
    for (int q = 0; q < QJ; ++q) acc[a][q] = 0.0;
  for (int k = 0; k < m; ++k) {
    double t[SP_RPT], s[QJ];
#pragma unroll
    for (int a = 0; a < SP_RPT; ++a) t[a] = T[(SP_RPT * ig + a) * tl + k];
#pragma unroll
    for (int q = 0; q < QJ; ++q) s[q] = S[k * mp + jg + 16 * q];
#pragma unroll
    for (int a = 0; a < SP_RPT; ++a)
#pragma unroll
      for (int q = 0; q < QJ; ++q) acc[a][q] += t[a] * s[q];
  }
}

// One pass along `axis` (0 x, 1 y, 2 z).  mode 0: out = S in along the axis;
// mode 1 (z only): out = S diag(1/Lambda) S in.
template <int QJ>
__global__ void __launch_bounds__(SP_NT)
k_spec_pass(const double* __restrict__ in, double* __restrict__ out, int nx, int ny, int nz, int axis, int mode,
            const double* __restrict__ Sg, int mp, const double* __restrict__ lx, const double* __restrict__ ly,
            const double* __restrict__ lz) {
  extern __shared__ double sp_sm[];
  const int m = axis == 0 ? nx : (axis == 1 ? ny : nz);
  const int tl = m + 1;              // padded tile row
  double* S = sp_sm;                 // [m][mp]
  double* T = sp_sm + (size_t)m * mp;  // [SP_W][tl]
  for (int e = threadIdx.x; e < m * mp; e += SP_NT) S[e] = Sg[e];
  const long nxy = (long)nx * ny;
  const int xt = (nx + SP_W - 1) / SP_W;
  const long ntile = axis == 0 ? ((long)ny * nz + SP_W - 1) / SP_W
                               : (axis == 1 ? (long)xt * nz : (nxy + SP_W - 1) / SP_W);
  const long is = axis == 0 ? nx : 1;           // stride between the lines of a tile
  const long as = axis == 0 ? 1 : (axis == 1 ? nx : nxy);  // stride along a line
  const int ig = threadIdx.x >> 4, jg = threadIdx.x & 15;
  for (long tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    long base;
    int w;
    if (axis == 0) {
      base = tile * SP_W * nx;
      w = (int)min((long)SP_W, (long)ny * nz - tile * SP_W);
    } else if (axis == 1) {
      const int x0 = (int)(tile % xt) * SP_W;
      base = x0 + nxy * (tile / xt);
      w = min(SP_W, nx - x0);
    } else {
      base = tile * SP_W;
      w = (int)min((long)SP_W, nxy - tile * SP_W);
    }
    __syncthreads();  // the previous tile's T is consumed (and S is loaded)
    // coalesced load: along the line for the x axis, across lines otherwise
    for (int e = threadIdx.x; e < SP_W * m; e += SP_NT) {
      int i, k;
      if (axis == 0) { i = e / m; k = e % m; }
      else { k = e / SP_W; i = e % SP_W; }
      T[i * tl + k] = i < w ? in[base + i * is + k * as] : 0.0;
    }
    __syncthreads();
    double acc[SP_RPT][QJ];
    sp_tile_mm<QJ>(T, tl, S, mp, m, acc);
    if (mode == 1) {
      // spectral coordinates: i -> (kx, ky) of the flat xy index, j -> kz
      __syncthreads();  // all reads of T done before it is overwritten
#pragma unroll
      for (int a = 0; a < SP_RPT; ++a) {
        const int i = SP_RPT * ig + a;
        const long qf = base + i;
        const double lxy = i < w ? lx[qf % nx] + ly[qf / nx] : 1.0;
#pragma unroll
        for (int q = 0; q < QJ; ++q) {
          const int j = jg + 16 * q;
          if (j < m) T[i * tl + j] = acc[a][q] / (lxy + lz[j]);
        }
      }
      __syncthreads();
      sp_tile_mm<QJ>(T, tl, S, mp, m, acc);
    }
    // store: thread (ig, jg) holds out[i][j]; write through shared memory so
    // the global stores are coalesced in the same order as the loads
    __syncthreads();
#pragma unroll
    for (int a = 0; a < SP_RPT; ++a)
#pragma unroll
      for (int q = 0; q < QJ; ++q) {
        const int j = jg + 16 * q;
        if (j < m) T[(SP_RPT * ig + a) * tl + j] = acc[a][q];
      }
    __syncthreads();
    for (int e = threadIdx.x; e < SP_W * m; e += SP_NT) {
      int i, k;
      if (axis == 0) { i = e / m; k = e % m; }
      else { k = e / SP_W; i = e % SP_W; }
      if (i < w) out[base + i * is + k * as] = T[i * tl + k];
    }
  }
}

static int spec_setup(psc_ctx* ctx) {
  if (ctx->spec_S[0]) return 0;
  const int dims[3] = {ctx->nx, ctx->ny, ctx->nz};
  for (int a = 0; a < 3; ++a) {
    const int m = dims[a];
    const int mp = 16 * ((m + 15) / 16);
    std::vector<double> S((size_t)m * mp, 0.0), lam(m);
    const double f = std::sqrt(2.0 / (m + 1));
    for (int j = 0; j < m; ++j)
      for (int k = 0; k < m; ++k) S[(size_t)k * mp + j] = f * std::sin(M_PI * (double)(j + 1) * (k + 1) / (m + 1));
    for (int k = 0; k < m; ++k) {
      const double th = M_PI * (k + 1) / (m + 1);
      double v = ctx->lap_c0 / 3.0;
      for (int d = 1; d <= 4; ++d) v += 2.0 * ctx->lap_c[d - 1] * std::cos(d * th);
      lam[k] = v;
    }
    PSC_CUDA(ctx, psc_dmalloc(&ctx->spec_S[a], S.size() * sizeof(double)));
    PSC_CUDA(ctx, psc_dmalloc(&ctx->spec_lam[a], lam.size() * sizeof(double)));
    PSC_CUDA(ctx, cudaMemcpy(ctx->spec_S[a], S.data(), S.size() * sizeof(double), cudaMemcpyHostToDevice));
    PSC_CUDA(ctx, cudaMemcpy(ctx->spec_lam[a], lam.data(), lam.size() * sizeof(double), cudaMemcpyHostToDevice));
    ctx->spec_mp[a] = mp;
  }
  if (!ctx->spec_tmp) PSC_CUDA(ctx, psc_dmalloc(&ctx->spec_tmp, 2 * ctx->n * sizeof(double)));
  return 0;
}

static int spec_pass(psc_ctx* ctx, const double* in, double* out, int axis, int mode, cudaStream_t st) {
  const int dims[3] = {ctx->nx, ctx->ny, ctx->nz};
  const int m = dims[axis];
  const int mp = ctx->spec_mp[axis];
  const size_t smem = ((size_t)m * mp + (size_t)SP_W * (m + 1)) * sizeof(double);
  const long nxy = (long)ctx->nx * ctx->ny;
  const long ntile = axis == 0 ? ((long)ctx->ny * ctx->nz + SP_W - 1) / SP_W
                               : (axis == 1 ? (long)((ctx->nx + SP_W - 1) / SP_W) * ctx->nz : (nxy + SP_W - 1) / SP_W);
  const int grid = (int)std::min<long>(ntile, 148L * 3);
  const int qj = mp / 16;
#define PSC_SPEC(Q)                                                                                        \
  case Q:                                                                                                  \
    PSC_CUDA(ctx, cudaFuncSetAttribute(k_spec_pass<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    k_spec_pass<Q><<<grid, SP_NT, smem, st>>>(in, out, ctx->nx, ctx->ny, ctx->nz, axis, mode,              \
                                              ctx->spec_S[axis], mp, ctx->spec_lam[0], ctx->spec_lam[1],    \
                                              ctx->spec_lam[2]);                                            \
    break;
  switch (qj) {
    PSC_SPEC(1) PSC_SPEC(2) PSC_SPEC(3) PSC_SPEC(4) PSC_SPEC(5) PSC_SPEC(6) PSC_SPEC(7) PSC_SPEC(8)
    default: PSC_REQUIRE(ctx, false, "poisson preconditioner: grid dimension above 128");
  }
#undef PSC_SPEC
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

static int spec_apply(psc_ctx* ctx, const double* r, double* z, cudaStream_t st) {
  double* t0 = ctx->spec_tmp;
  double* t1 = ctx->spec_tmp + ctx->n;
  int rc = spec_pass(ctx, r, t0, 0, 0, st);
  if (!rc) rc = spec_pass(ctx, t0, t1, 1, 0, st);
  if (!rc) rc = spec_pass(ctx, t1, t0, 2, 1, st);
  if (!rc) rc = spec_pass(ctx, t0, t1, 1, 0, st);
  if (!rc) rc = spec_pass(ctx, t1, z, 0, 0, st);
  return rc;
}

extern "C" int psc_poisson_precond(psc_ctx* ctx, const double* r, double* z, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, r && z && r != z, "poisson_precond: bad arguments");
  PSC_REQUIRE(ctx, ctx->nx <= SP_MAXM && ctx->ny <= SP_MAXM && ctx->nz <= SP_MAXM,
              "poisson preconditioner: grid dimension above 128");
  if (spec_setup(ctx)) return 1;
  return spec_apply(ctx, r, z, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// preconditioned CG; scalars on the device, the host reads z.r once per
// iteration for the stop test (these solves take about ten iterations)
// ---------------------------------------------------------------------------
constexpr int PCG_NT = 256;

// alpha = ro / p.Ap (sum of the stencil's per-block partials, fixed order);
// x += alpha p; r -= alpha Ap
__global__ void __launch_bounds__(PCG_NT)
k_pcg_step(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
           const double* __restrict__ ap, long n, const double* __restrict__ part, int np, const double* sc) {
  __shared__ double sh[PCG_NT / 32];
  __shared__ double bc;
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += PCG_NT) s += part[i];
  s = psc_block_sum<double, PCG_NT>(s, sh);
  if (threadIdx.x == 0) bc = s;
  __syncthreads();
  const double alp = sc[0] / bc;
  for (long i = blockIdx.x * (long)PCG_NT + threadIdx.x; i < n; i += (long)gridDim.x * PCG_NT) {
    x[i] += alp * p[i];
    r[i] -= alp * ap[i];
  }
}

// p = z + (ro1 / ro) p
__global__ void k_pcg_dir(const double* __restrict__ z, double* __restrict__ p, long n, const double* sc) {
  const double bet = sc[1] / sc[0];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    p[i] = z[i] + bet * p[i];
}

__global__ void k_pcg_shift(double* sc) {
  if (threadIdx.x == 0 && blockIdx.x == 0) sc[0] = sc[1];
}

extern "C" int psc_pcg_poisson_prec(psc_ctx* ctx, const double* rhs, double* x, int maxit, double tol, int* its_out,
                                    void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, rhs && x && maxit >= 0, "pcg_prec: bad arguments");
  PSC_REQUIRE(ctx, ctx->nx <= SP_MAXM && ctx->ny <= SP_MAXM && ctx->nz <= SP_MAXM,
              "poisson preconditioner: grid dimension above 128");
  cudaStream_t st = (cudaStream_t)stream;
  if (spec_setup(ctx)) return 1;
  const long n = ctx->n;
  if (!ctx->cg_x) PSC_CUDA(ctx, psc_dmalloc(&ctx->cg_x, n * sizeof(double)));
  if (!ctx->cg_p2) PSC_CUDA(ctx, psc_dmalloc(&ctx->cg_p2, n * sizeof(double)));
  double* r = ctx->cg_r;
  double* p = ctx->cg_p;
  double* ap = ctx->cg_ap;
  double* z = ctx->cg_p2;
  double* sc = ctx->scalars + 96;   // [0] ro, [1] ro1 (this solve's slots)
  // partials of the fused stencil: one per block of its launch
  const int need = std::max(PSC_RED_BLOCKS, psc_stencil_blocks(ctx, 1));
  if (ctx->cg_part_cap < need) {
    psc_dfree(ctx->cg_part);
    ctx->cg_part = nullptr;
    PSC_CUDA(ctx, psc_dmalloc(&ctx->cg_part, 2 * (size_t)need * sizeof(double)));
    ctx->cg_part_cap = need;
  }
  // r = rhs - A x; z = M r; p = z; ro1 = z.r
  int rc = psc_laplacian_fused(ctx, x, rhs, r, -1.0, 0.0, 1.0, nullptr, nullptr, st);
  if (rc) return rc;
  rc = spec_apply(ctx, r, z, st);
  if (rc) return rc;
  PSC_CUDA(ctx, cudaMemcpyAsync(p, z, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  const double* za[1] = {z};
  const double* ra[1] = {r};
  rc = psc_dots(ctx, 1, za, ra, n, sc + 1, st);
  if (rc) return rc;
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->host_scalars + 96, sc + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  double ro1 = ctx->host_scalars[96];
  const double tol1 = tol * tol * ro1;
  int its = 0;
  const int nb = 148 * 4;
  while (its < maxit && ro1 > tol1) {
    ++its;
    k_pcg_shift<<<1, 32, 0, st>>>(sc);                 // ro = ro1
    PSC_LAUNCH_CHECK(ctx);
    int nblk = 0;
    rc = psc_laplacian_fused(ctx, p, nullptr, ap, 1.0, 0.0, 0.0, ctx->cg_part, &nblk, st);   // Ap, p.Ap partials
    if (rc) return rc;
    k_pcg_step<<<nb, PCG_NT, 0, st>>>(x, r, p, ap, n, ctx->cg_part, nblk, sc);
    PSC_LAUNCH_CHECK(ctx);
    rc = spec_apply(ctx, r, z, st);
    if (rc) return rc;
    rc = psc_dots(ctx, 1, za, ra, n, sc + 1, st);
    if (rc) return rc;
    k_pcg_dir<<<nb, 256, 0, st>>>(z, p, n, sc);
    PSC_LAUNCH_CHECK(ctx);
    PSC_CUDA(ctx, cudaMemcpyAsync(ctx->host_scalars + 96, sc + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    PSC_CUDA(ctx, cudaStreamSynchronize(st));
    ro1 = ctx->host_scalars[96];
  }
  if (its_out) *its_out = its;
  return 0;
}
