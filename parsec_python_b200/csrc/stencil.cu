// Matrix-free Hamiltonian / Laplacian application and the Chebyshev filter.
//
// One launch computes, for a block of k column vectors,
//   Out = alpha * (W * In) + beta * In + gamma * Prev
// where W is either the Hamiltonian's local part 0.5*A + diag(pot) or the
// Laplacian A = -Lap_h alone (pot == NULL).  The Kleinman-Bylander term is
// added by nonlocal.cu (project before, scatter after).
//
// Kernel shape (B200): each CTA owns a contiguous slab of S = 256*PPT flat xy
// points of one column and marches in z over a chunk of planes.  The 2R+1
// z-neighbours of each owned point are kept in a register queue; the current
// plane (owned points + R rows of y halo on each side) is staged in shared
// memory, double buffered, so x and y neighbours come from shared memory and
// every global load is a coalesced row segment.  HBM traffic per step is one
// read of In, one read of Prev and one write of Out per point and column.
#include "psc_internal.cuh"
#include "../../include/psc.h"

template <typename T>
struct StencilW {
  T c0;      // centre weight
  T c[4];    // offset weights
};

template <typename T, int R, int PPT>
__global__ void __launch_bounds__(256)
k_stencil(const T* __restrict__ X, long ldx, const T* Pv, long ldp, T* Y, long ldy,
          const T* __restrict__ pot, int nx, int ny, int nz, int zchunk, StencilW<T> w,
          const double* __restrict__ coef, double ha, double hb, double hg,
          double* __restrict__ dot_partial) {
  constexpr int NT = 256;
  constexpr int S = NT * PPT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* plane = reinterpret_cast<T*>(smem_raw);
  const int nxy = nx * ny;
  const int halo = R * nx;
  const int win = S + 2 * halo;           // window length per buffer
  const int slab0 = blockIdx.x * S;
  const int seff = min(S, nxy - slab0);   // owned points in this slab
  const int z0 = blockIdx.y * zchunk;
  const int z1 = min(nz, z0 + zchunk);
  const long col = blockIdx.z;
  const T* Xc = X + col * ldx;
  const T* Pc = Pv ? Pv + col * ldp : nullptr;
  T* Yc = Y + col * ldy;

  T a, b, g;
  if (coef) { a = (T)coef[0]; b = (T)coef[1]; g = (T)coef[2]; }
  else { a = (T)ha; b = (T)hb; g = (T)hg; }

  int q[PPT], xi[PPT], yi[PPT];
  bool own[PPT];
#pragma unroll
  for (int v = 0; v < PPT; ++v) {
    const int loc = threadIdx.x + NT * v;
    own[v] = loc < seff;
    q[v] = slab0 + loc;
    xi[v] = own[v] ? q[v] % nx : 0;
    yi[v] = own[v] ? q[v] / nx : 0;
  }

  // z queue: zq[v][i] holds plane z - R + i of owned point v.
  T zq[PPT][2 * R + 1];
#pragma unroll
  for (int v = 0; v < PPT; ++v)
#pragma unroll
    for (int i = 0; i < 2 * R; ++i) {
      const int zz = z0 - R + i;
      zq[v][i] = (own[v] && zz >= 0 && zz < nz) ? Xc[(long)zz * nxy + q[v]] : T(0);
    }

  double dacc = 0.0;
  int buf = 0;
  const int hcount = win - seff;          // non-owned window positions
  for (int z = z0; z < z1; ++z) {
    T* pl = plane + buf * win;
    const long zoff = (long)z * nxy;
#pragma unroll
    for (int v = 0; v < PPT; ++v) {
      const int zz = z + R;
      zq[v][2 * R] = (own[v] && zz < nz) ? Xc[(long)zz * nxy + q[v]] : T(0);
      if (own[v]) pl[halo + threadIdx.x + NT * v] = zq[v][R];
    }
    for (int j = threadIdx.x; j < hcount; j += NT) {
      const int pos = j < halo ? j : j + seff;
      const int fq = slab0 - halo + pos;
      pl[pos] = (fq >= 0 && fq < nxy) ? Xc[zoff + fq] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < PPT; ++v) {
      if (!own[v]) continue;
      const int s = halo + threadIdx.x + NT * v;
      const T xc = zq[v][R];
      T acc = w.c0 * xc;
#pragma unroll
      for (int d = 1; d <= R; ++d) {
        const T cd = w.c[d - 1];
        T sx = T(0), sy = T(0), sz = T(0);
        if (xi[v] - d >= 0) sx += pl[s - d];
        if (xi[v] + d < nx) sx += pl[s + d];
        if (yi[v] - d >= 0) sy += pl[s - d * nx];
        if (yi[v] + d < ny) sy += pl[s + d * nx];
        sz = zq[v][R - d] + zq[v][R + d];
        acc += cd * (sx + sy + sz);
      }
      if (pot) acc += pot[zoff + q[v]] * xc;
      T out = a * acc + b * xc;
      if (Pc) out += g * Pc[zoff + q[v]];
      Yc[zoff + q[v]] = out;
      if (dot_partial) dacc += (double)out * (double)xc;
    }
#pragma unroll
    for (int v = 0; v < PPT; ++v)
#pragma unroll
      for (int i = 0; i < 2 * R; ++i) zq[v][i] = zq[v][i + 1];
    buf ^= 1;
  }
  if (dot_partial) {
    __shared__ double sh[NT / 32];
    dacc = psc_block_sum<double, NT>(dacc, sh);
    if (threadIdx.x == 0)
      dot_partial[((long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = dacc;
  }
}

struct StencilPlan {
  int ppt, zchunk;
  dim3 grid;
  size_t smem;
};

// Choose points-per-thread and z-chunk so that the grid holds a few CTAs per
// SM even for a single column, with long z runs when there are many columns.
static StencilPlan plan_stencil(const psc_ctx* ctx, int k, size_t elem) {
  StencilPlan p;
  const int nxy = ctx->nx * ctx->ny;
  p.ppt = (nxy >= 2048) ? 2 : 1;
  const int S = 256 * p.ppt;
  const int nslab = (nxy + S - 1) / S;
  const long target = 148L * 6;
  long per_col = (target + k - 1) / k;
  int nzc = (int)std::max<long>(1, std::min<long>(ctx->nz, (per_col + nslab - 1) / nslab));
  int zchunk = (ctx->nz + nzc - 1) / nzc;
  if (zchunk < 4) zchunk = std::min(ctx->nz, 4);
  nzc = (ctx->nz + zchunk - 1) / zchunk;
  p.zchunk = zchunk;
  p.grid = dim3(nslab, nzc, k);
  p.smem = 2 * (size_t)(S + 2 * ctx->radius * ctx->nx) * elem;
  return p;
}

template <typename T, int R, int PPT>
static int launch_stencil_t(psc_ctx* ctx, const StencilPlan& p, const T* X, long ldx, const T* P,
                            long ldp, T* Y, long ldy, const T* pot, StencilW<T> w, const double* coef,
                            double a, double b, double g, double* dot_partial, cudaStream_t st) {
  auto kern = k_stencil<T, R, PPT>;
  if (p.smem > 40 * 1024) {
    PSC_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem));
  }
  kern<<<p.grid, 256, p.smem, st>>>(X, ldx, P, ldp, Y, ldy, pot, ctx->nx, ctx->ny, ctx->nz, p.zchunk, w,
                                    coef, a, b, g, dot_partial);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

template <typename T>
int psc_stencil_tma(psc_ctx* ctx, int k, const T* X, long ldx, const T* P, long ldp, T* Y, long ldy, const T* pot,
                    const double* w, const double* coef, double a, double b, double g, bool masked,
                    cudaStream_t st);

// Sphere mask: zero every point of k columns farther than sqrt(mask_r2)
// from the cube's centre.
template <typename T>
__global__ void k_apply_mask(T* X, long ld, int k, int nx, int ny, long n, double h, double cx, double cy, double cz,
                             double r2) {
  const long total = n * (long)k;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long p = e % n;
    const int c = (int)(e / n);
    const double x = (p % nx) * h - cx, y = ((p / nx) % ny) * h - cy, z = (p / ((long)nx * ny)) * h - cz;
    if (x * x + y * y + z * z > r2) X[p + (long)c * ld] = T(0);
  }
}

int psc_mask_block_impl(psc_ctx* ctx, int dtype, void* X, long ld, int k, cudaStream_t st) {
  if (ctx->mask_r2 <= 0.0 || k < 1) return 0;
  const long total = ctx->n * (long)k;
  const int nb = (int)std::min<long>(148L * 16, (total + 255) / 256);
  if (dtype == PSC_F64)
    k_apply_mask<double><<<nb, 256, 0, st>>>((double*)X, ld, k, ctx->nx, ctx->ny, ctx->n, ctx->h, ctx->mask_c[0],
                                             ctx->mask_c[1], ctx->mask_c[2], ctx->mask_r2);
  else
    k_apply_mask<float><<<nb, 256, 0, st>>>((float*)X, ld, k, ctx->nx, ctx->ny, ctx->n, ctx->h, ctx->mask_c[0],
                                            ctx->mask_c[1], ctx->mask_c[2], ctx->mask_r2);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

template <typename T>
static int launch_stencil(psc_ctx* ctx, int k, const T* X, long ldx, const T* P, long ldp, T* Y, long ldy,
                          const T* pot, const double* c0c, const double* coef, double a, double b,
                          double g, double* dot_partial, int* nblocks_out, cudaStream_t st, bool masked = false) {
  // the TMA pipeline serves every launch that needs no fused dot product and
  // meets the bulk-copy alignment rules; the register-queue kernel the rest
  // (followed by a masking pass when the Hamiltonian is sphere-masked)
  if (!dot_partial && ctx->stencil_impl != 1) {
    const int rc = psc_stencil_tma<T>(ctx, k, X, ldx, P, ldp, Y, ldy, pot, c0c, coef, a, b, g, masked, st);
    if (rc >= 0) return rc;
  }
  if (masked && ctx->mask_r2 > 0.0) {
    const int rc = launch_stencil<T>(ctx, k, X, ldx, P, ldp, Y, ldy, pot, c0c, coef, a, b, g, dot_partial,
                                     nblocks_out, st, false);
    if (rc) return rc;
    return psc_mask_block_impl(ctx, sizeof(T) == 8 ? PSC_F64 : PSC_F32, Y, ldy, k, st);
  }
  StencilPlan p = plan_stencil(ctx, k, sizeof(T));
  if (nblocks_out) *nblocks_out = (int)(p.grid.x * p.grid.y * p.grid.z);
  StencilW<T> w;
  w.c0 = (T)c0c[0];
  for (int i = 0; i < 4; ++i) w.c[i] = (T)c0c[1 + i];
  const int R = ctx->radius;
#define PSC_DISPATCH(RR)                                                                           \
  if (R == RR) {                                                                                   \
    if (p.ppt == 2)                                                                                \
      return launch_stencil_t<T, RR, 2>(ctx, p, X, ldx, P, ldp, Y, ldy, pot, w, coef, a, b, g,     \
                                        dot_partial, st);                                         \
    return launch_stencil_t<T, RR, 1>(ctx, p, X, ldx, P, ldp, Y, ldy, pot, w, coef, a, b, g,       \
                                      dot_partial, st);                                           \
  }
  PSC_DISPATCH(1) PSC_DISPATCH(2) PSC_DISPATCH(3) PSC_DISPATCH(4)
#undef PSC_DISPATCH
  PSC_REQUIRE(ctx, false, "stencil radius must be 1..4");
}

int psc_stencil_blocks(psc_ctx* ctx, int k) {
  StencilPlan p = plan_stencil(ctx, k, sizeof(double));
  return (int)(p.grid.x * p.grid.y * p.grid.z);
}

// Laplacian (k = 1, double) with an optional fused per-block partial of Out.In.
int psc_laplacian_fused(psc_ctx* ctx, const double* x, const double* prev, double* y, double a, double b,
                        double g, double* dot_partial, int* nblocks, cudaStream_t st) {
  double w[5] = {ctx->lap_c0, ctx->lap_c[0], ctx->lap_c[1], ctx->lap_c[2], ctx->lap_c[3]};
  return launch_stencil<double>(ctx, 1, x, ctx->n, prev, ctx->n, y, ctx->n, nullptr, w, nullptr, a, b, g,
                                dot_partial, nblocks, st);
}

// nonlocal.cu
int psc_nl_project(psc_ctx* ctx, int dtype, const void* X, long ldx, int k, cudaStream_t st);
int psc_nl_scatter(psc_ctx* ctx, int dtype, void* Y, long ldy, int k, const double* coef, double a,
                   cudaStream_t st);

int psc_apply_h_impl(psc_ctx* ctx, int dtype, const void* X, long ldx, void* Y, long ldy, const void* P,
                     long ldp, int k, const double* coef_dev, double a, double b, double g,
                     cudaStream_t st) {
  PSC_REQUIRE(ctx, k >= 1 && k <= 65535, "apply_h: k out of range");
  PSC_REQUIRE(ctx, ldx >= ctx->n && ldy >= ctx->n && (!P || ldp >= ctx->n), "apply_h: ld < n");
  PSC_REQUIRE(ctx, X != Y, "apply_h: input and output must differ");
  if (ctx->nl_atoms > 0) {
    int rc = psc_nl_project(ctx, dtype, X, ldx, k, st);
    if (rc) return rc;
  }
  double w[5] = {ctx->ham_c0, ctx->ham_c[0], ctx->ham_c[1], ctx->ham_c[2], ctx->ham_c[3]};
  int rc;
  if (dtype == PSC_F64)
    rc = launch_stencil<double>(ctx, k, (const double*)X, ldx, (const double*)P, ldp, (double*)Y, ldy,
                                ctx->pot64, w, coef_dev, a, b, g, nullptr, nullptr, st, true);
  else
    rc = launch_stencil<float>(ctx, k, (const float*)X, ldx, (const float*)P, ldp, (float*)Y, ldy,
                               ctx->pot32, w, coef_dev, a, b, g, nullptr, nullptr, st, true);
  if (rc) return rc;
  if (ctx->nl_atoms > 0) return psc_nl_scatter(ctx, dtype, Y, ldy, k, coef_dev, a, st);
  return 0;
}

// Y = V_nl X alone (the factored Kleinman-Bylander term), for checks against
// the reference's V_nl matrix without the Laplacian around it.
extern "C" int psc_apply_nonlocal(psc_ctx* ctx, int dtype, const void* X, long ldx, void* Y, long ldy, int k,
                                  void* stream) {
  if (!ctx) return 2;
  cudaStream_t st = (cudaStream_t)stream;
  PSC_REQUIRE(ctx, X && Y && X != Y && k >= 1 && ldx >= ctx->n && ldy >= ctx->n, "apply_nonlocal: bad arguments");
  const size_t es = dtype == PSC_F64 ? sizeof(double) : sizeof(float);
  PSC_CUDA(ctx, cudaMemset2DAsync(Y, ldy * es, 0, ctx->n * es, k, st));
  if (ctx->nl_atoms == 0) return 0;
  int rc = psc_nl_project(ctx, dtype, X, ldx, k, st);
  if (rc) return rc;
  return psc_nl_scatter(ctx, dtype, Y, ldy, k, nullptr, 1.0, st);
}

extern "C" int psc_apply_h(psc_ctx* ctx, int dtype, const void* X, long ldx, void* Y, long ldy, int k,
                           void* stream) {
  if (!ctx) return 2;
  return psc_apply_h_impl(ctx, dtype, X, ldx, Y, ldy, nullptr, 0, k, nullptr, 1.0, 0.0, 0.0,
                          (cudaStream_t)stream);
}

extern "C" int psc_apply_h_axpby(psc_ctx* ctx, int dtype, const void* X, long ldx, const void* P, long ldp,
                                 void* Y, long ldy, int k, double alpha, double beta, double gamma,
                                 void* stream) {
  if (!ctx) return 2;
  return psc_apply_h_impl(ctx, dtype, X, ldx, Y, ldy, P, ldp, k, nullptr, alpha, beta, gamma,
                          (cudaStream_t)stream);
}

extern "C" int psc_laplacian_apply(psc_ctx* ctx, const double* x, double* y, int k, long ld, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, x != y && ld >= ctx->n, "laplacian_apply: bad arguments");
  double w[5] = {ctx->lap_c0, ctx->lap_c[0], ctx->lap_c[1], ctx->lap_c[2], ctx->lap_c[3]};
  return launch_stencil<double>(ctx, k, x, ld, nullptr, 0, y, ld, nullptr, w, nullptr, 1.0, 0.0, 0.0,
                                nullptr, nullptr, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Chebyshev filter coefficients computed on the device from device bounds.
// mode 0 = scaled filter (Eigensolvers/ch_filter.py:4-81),
// mode 1 = slim filter  (Eigensolvers/first_filt.py:78-103).
// bounds = [lam1, low, high].  coef[j] = (alpha, beta, gamma) of step j.
// ---------------------------------------------------------------------------
__global__ void k_cheb_coef(int mode, int deg, const double* bounds, double* coef, int* status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double lam1 = bounds[0], lo = bounds[1], hi = bounds[2];
  const double e = (hi - lo) / 2;
  const double c = (hi + lo) / 2;
  if (!(hi > lo)) status[0] = 1;  // bounds are incorrect (chefsi1.py:37-38)
  if (mode == 0) {
    const double s1 = e / (lam1 - c);
    double s = s1;
    coef[0] = s1 / e;
    coef[1] = -c * (s1 / e);
    coef[2] = 0.0;
    const double two_s1 = 2.0 / s1;
    const double inv_e = 1.0 / e;
    for (int j = 1; j < deg; ++j) {
      const double sn = 1.0 / (two_s1 - s);
      const double t1 = 2.0 * sn * inv_e;
      const double t2 = s * sn;
      coef[3 * j + 0] = t1;
      coef[3 * j + 1] = -c * t1;
      coef[3 * j + 2] = -t2;
      s = sn;
    }
  } else {
    coef[0] = -1.0 / e;
    coef[1] = c / e;
    coef[2] = 0.0;
    for (int j = 1; j < deg; ++j) {
      coef[3 * j + 0] = -2.0 / e;
      coef[3 * j + 1] = 2.0 * c / e;
      coef[3 * j + 2] = -1.0;
    }
  }
}

// Filter X (k columns) to degree deg.  X holds Y_0 on entry and is reused as
// storage, Y is the second buffer; *which = 0 if the result is in X, 1 if in Y.
extern "C" int psc_cheb_filter(psc_ctx* ctx, int dtype, int mode, int deg, const double* bounds_dev,
                               void* X, void* Y, long ld, int k, int* which, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, deg >= 1 && deg <= PSC_MAX_DEG, "cheb_filter: degree out of range");
  PSC_REQUIRE(ctx, mode == 0 || mode == 1, "cheb_filter: mode must be 0 (scaled) or 1 (slim)");
  cudaStream_t st = (cudaStream_t)stream;
  k_cheb_coef<<<1, 32, 0, st>>>(mode, deg, bounds_dev, ctx->cheb_coef, ctx->dev_status);
  PSC_LAUNCH_CHECK(ctx);
  void* buf[2] = {X, Y};
  // step 0: Y = a*H X + b*X
  int rc = psc_apply_h_impl(ctx, dtype, X, ld, Y, ld, nullptr, 0, k, ctx->cheb_coef, 0, 0, 0, st);
  if (rc) return rc;
  int cur = 1;  // buffer holding Y_j
  for (int j = 1; j < deg; ++j) {
    // Y_{j+1} = a*H Y_j + b*Y_j + g*Y_{j-1}, written over Y_{j-1}
    rc = psc_apply_h_impl(ctx, dtype, buf[cur], ld, buf[cur ^ 1], ld, buf[cur ^ 1], ld, k,
                          ctx->cheb_coef + 3 * j, 0, 0, 0, st);
    if (rc) return rc;
    cur ^= 1;
  }
  if (which) *which = cur;
  return 0;
}

// 0: TMA pipeline wherever it applies (default), 1: register-queue kernel only.
// Sphere-masked Hamiltonian: H X = P (0.5 A + V_nl + diag(pot)) X with P
// zeroing the points farther than `radius` (bohr) from the cube's centre;
// radius <= 0 restores the cube.  The projector tables lose their points
// outside the sphere.  Meant for blocks that vanish outside the sphere (the
// solver masks its random start); there the masked operator is P H P.
int psc_nl_apply_mask(psc_ctx* ctx, cudaStream_t st);
extern "C" int psc_set_sphere_mask(psc_ctx* ctx, double radius, void* stream) {
  if (!ctx) return 2;
  ctx->mask_r2 = radius > 0.0 ? radius * radius : 0.0;
  ctx->mask_c[0] = 0.5 * ctx->h * (ctx->nx - 1);
  ctx->mask_c[1] = 0.5 * ctx->h * (ctx->ny - 1);
  ctx->mask_c[2] = 0.5 * ctx->h * (ctx->nz - 1);
  // masked work tables depend on the radius: drop the cached ones once the
  // launches that may still read them have finished
  PSC_CUDA(ctx, cudaStreamSynchronize((cudaStream_t)stream));
  for (auto& e : ctx->st_sched) psc_dfree(e.dev);
  ctx->st_sched.clear();
  return psc_nl_apply_mask(ctx, (cudaStream_t)stream);
}

extern "C" int psc_mask_block(psc_ctx* ctx, int dtype, void* X, long ld, int k, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, X && ld >= ctx->n && k >= 0, "mask_block: bad arguments");
  return psc_mask_block_impl(ctx, dtype, X, ld, k, (cudaStream_t)stream);
}

int psc_recast_pot32(psc_ctx* ctx, cudaStream_t st);

extern "C" int psc_set_stencil_weights(psc_ctx* ctx, int mode) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, mode >= 0 && mode <= 2, "stencil weights mode must be 0, 1 or 2");
  ctx->stencil_comp = mode;
  // pot32 follows the mode (it carries the correction in mode 2 only); the
  // legacy default stream orders this after work queued on blocking streams
  if (int rc = psc_recast_pot32(ctx, nullptr)) return rc;
  PSC_CUDA(ctx, cudaStreamSynchronize(nullptr));
  return 0;
}

extern "C" int psc_set_stencil_impl(psc_ctx* ctx, int impl) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, impl >= 0 && impl <= 4, "stencil impl must be 0 .. 4");
  ctx->stencil_impl = impl;
  return 0;
}
