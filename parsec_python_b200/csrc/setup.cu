// Ionic setup kernels: SAD density, local pseudopotential and SAD Hartree
// potential (V_ion/pseudoDiag.py:44-421), projector ball geometry and values
// (V_ion/pseudoNL_original.py:115-196), and a NumPy-order pairwise sum.
//
// This translation unit is compiled with --fmad=false: every product and sum
// is rounded separately, in the reference's operation order, so the SAD
// fields come out bit-identical to the reference's CPU code.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <cmath>
#include <vector>

__device__ __forceinline__ double spline_eval(const psc_spline_dev s, double x) {
  // Splines/fsplevalIO.py:2-65: clamp to the knot range, locate the interval
  // by bisection (largest j with xi[j] <= x, at most n-2), evaluate.
  const double* xi = s.x;
  const int n = s.n;
  if (x < xi[0]) x = xi[0];
  else if (x > xi[n - 1]) x = xi[n - 1];
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int mid = (hi + lo) >> 1;
    if (x < xi[mid]) hi = mid;
    else lo = mid;
  }
  const int j = lo;
  const double t1 = xi[j + 1] - x;
  const double t2 = x - xi[j];
  const double hj = xi[j + 1] - xi[j];
  return t1 * (s.z[j] * t1 * t1 / hj + s.c[j]) + t2 * (s.z[j + 1] * t2 * t2 / hj + s.d[j]);
}

__global__ void k_sad(int nx, int ny, int nz, double h, double rad, int natoms, const int* __restrict__ sp,
                      const double* __restrict__ xyz, const psc_spline_dev* __restrict__ tab, double h3,
                      double fourpi, double* __restrict__ rho0, double* __restrict__ hpot0,
                      double* __restrict__ ppot) {
  const long n = (long)nx * ny * nz;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x) {
    const int i = (int)(p % nx);
    const int j = (int)((p / nx) % ny);
    const int k = (int)(p / ((long)nx * ny));
    double pv = 0.0, rv = 0.0, hv = 0.0;
    for (int a = 0; a < natoms; ++a) {
      const double dz = (double)k * h - rad - xyz[3 * a + 2];
      const double dy = (double)j * h - rad - xyz[3 * a + 1];
      const double dx = (double)i * h - rad - xyz[3 * a + 0];
      const double r = sqrt((dz * dz + dy * dy) + dx * dx);
      const psc_spline_dev* t = tab + 5 * sp[a];
      pv += spline_eval(t[2], r);
      const double rr = spline_eval(t[0], r) * h3 / fourpi;
      rv += (rr > 0.0) ? rr : 0.0;
      hv += spline_eval(t[1], r);
    }
    rho0[p] = rv;
    hpot0[p] = hv;
    ppot[p] = pv;
  }
}

__global__ void k_scale_div(double* x, long n, const double* num_scalar, double znum, const double* den) {
  // x <- znum * x / den  (pseudoDiag.py:296: rho0 = Z_sum * rho0 / rho0_sum)
  const double d = *den;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < n; p += (long)gridDim.x * blockDim.x)
    x[p] = znum * x[p] / d;
}

// ---------------------------------------------------------------------------
// NumPy's pairwise summation (the order np.sum uses for a contiguous float64
// vector): blocks of <= 128 elements summed with 8 interleaved accumulators,
// blocks of < 8 summed sequentially, larger ranges split at n/2 rounded down
// to a multiple of 8.  Leaves are summed in parallel; the recursion above
// them is a fixed binary tree, built on the host once per length and
// evaluated level by level in one CTA (each node the sum of its left and
// right child, so every addition is the one np.sum makes).
// ---------------------------------------------------------------------------
namespace {
// the node of range [off, off + n): -(leaf index + 1) for a leaf, else the
// index of an internal node; appends the leaves and the internal nodes below
// it, with each internal node's height above the leaves
int pw_build(long off, long n, std::vector<long>& lo, std::vector<long>& len, std::vector<int2>& kids,
             std::vector<int>& height) {
  if (n <= 128) {
    lo.push_back(off);
    len.push_back(n);
    return -(int)lo.size();
  }
  long n2 = n / 2;
  n2 -= n2 % 8;
  const int a = pw_build(off, n2, lo, len, kids, height);
  const int b = pw_build(off + n2, n - n2, lo, len, kids, height);
  kids.push_back(make_int2(a, b));
  const int ha = a < 0 ? 0 : height[a], hb = b < 0 ? 0 : height[b];
  height.push_back(1 + std::max(ha, hb));
  return (int)kids.size() - 1;
}
}  // namespace

__global__ void k_pw_leaf(const double* __restrict__ a, const long* __restrict__ lo, const long* __restrict__ len,
                          long nleaf, double* __restrict__ out) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < nleaf; t += (long)gridDim.x * blockDim.x) {
    const double* x = a + lo[t];
    const long n = len[t];
    double res;
    if (n < 8) {
      res = 0.0;
      for (long i = 0; i < n; ++i) res += x[i];
    } else {
      double r[8];
      for (int j = 0; j < 8; ++j) r[j] = x[j];
      long i = 8;
      for (; i < n - (n % 8); i += 8)
        for (int j = 0; j < 8; ++j) r[j] += x[i + j];
      res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
      for (; i < n; ++i) res += x[i];
    }
    out[t] = res;
  }
}

// vals[0, nleaf) = leaf sums; internal node i lands in vals[nleaf + i].
// order[] lists the internal nodes level by level (level_off[h] .. level_off[h+1]).
__global__ void __launch_bounds__(1024) k_pw_tree(const int2* __restrict__ kids, const int* __restrict__ order,
                                                   const int* __restrict__ level_off, int nlevel, int nleaf,
                                                   double* vals, double* out) {
  for (int h = 0; h < nlevel; ++h) {
    for (int t = level_off[h] + threadIdx.x; t < level_off[h + 1]; t += blockDim.x) {
      const int i = order[t];
      const int2 c = kids[i];
      const double a = vals[c.x < 0 ? -c.x - 1 : nleaf + c.x];
      const double b = vals[c.y < 0 ? -c.y - 1 : nleaf + c.y];
      vals[nleaf + i] = a + b;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = nlevel ? vals[nleaf + order[level_off[nlevel] - 1]] : vals[0];
}

extern "C" int psc_numpy_sum(psc_ctx* ctx, const double* x, long n, double* out_dev, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, n >= 1, "numpy_sum: n < 1");
  cudaStream_t st = (cudaStream_t)stream;
  if (ctx->pw_n != n) {
    std::vector<long> lo, len;
    std::vector<int2> kids;
    std::vector<int> height;
    pw_build(0, n, lo, len, kids, height);
    const int nl = (int)lo.size(), ni = (int)kids.size();
    int nlevel = 0;
    for (int hgt : height) nlevel = std::max(nlevel, hgt);
    // internal nodes ordered by height: those of height h + 1 at off[h] .. off[h + 1]
    std::vector<int> cnt(nlevel + 1, 0), off(nlevel + 1, 0), order(std::max(ni, 1));
    for (int hgt : height) ++cnt[hgt];
    for (int h = 1; h <= nlevel; ++h) off[h] = off[h - 1] + cnt[h];
    std::vector<int> fill(off.begin(), off.end());
    for (int i = 0; i < ni; ++i) order[fill[height[i] - 1]++] = i;
    psc_dfree(ctx->pw_buf);
    ctx->pw_buf = nullptr;
    ctx->pw_n = 0;
    // one allocation: lo, len (long), leaf + node sums (double), kids (int2), order, level offsets (int)
    const size_t bytes = (size_t)nl * 8 * 2 + (size_t)(nl + ni) * 8 + (size_t)std::max(ni, 1) * 8 +
                         (size_t)std::max(ni, 1) * 4 + (size_t)(nlevel + 1) * 4 + 64;
    PSC_CUDA(ctx, psc_dmalloc(&ctx->pw_buf, bytes));
    char* b = static_cast<char*>(ctx->pw_buf);
    ctx->pw_lo = reinterpret_cast<long*>(b);
    ctx->pw_len = ctx->pw_lo + nl;
    ctx->pw_vals = reinterpret_cast<double*>(ctx->pw_len + nl);
    ctx->pw_kids = reinterpret_cast<int2*>(ctx->pw_vals + nl + ni);
    ctx->pw_order = reinterpret_cast<int*>(ctx->pw_kids + std::max(ni, 1));
    ctx->pw_level_off = ctx->pw_order + std::max(ni, 1);
    PSC_CUDA(ctx, cudaMemcpy(ctx->pw_lo, lo.data(), nl * sizeof(long), cudaMemcpyHostToDevice));
    PSC_CUDA(ctx, cudaMemcpy(ctx->pw_len, len.data(), nl * sizeof(long), cudaMemcpyHostToDevice));
    if (ni) {
      PSC_CUDA(ctx, cudaMemcpy(ctx->pw_kids, kids.data(), ni * sizeof(int2), cudaMemcpyHostToDevice));
      PSC_CUDA(ctx, cudaMemcpy(ctx->pw_order, order.data(), ni * sizeof(int), cudaMemcpyHostToDevice));
    }
    PSC_CUDA(ctx, cudaMemcpy(ctx->pw_level_off, off.data(), (nlevel + 1) * sizeof(int), cudaMemcpyHostToDevice));
    ctx->pw_nleaf = nl;
    ctx->pw_nlevel = nlevel;
    ctx->pw_n = n;
  }
  const long nl = ctx->pw_nleaf;
  k_pw_leaf<<<std::max(1, (int)std::min<long>(1184, (nl + 127) / 128)), 128, 0, st>>>(x, ctx->pw_lo, ctx->pw_len,
                                                                                   nl, ctx->pw_vals);
  PSC_LAUNCH_CHECK(ctx);
  k_pw_tree<<<1, 1024, 0, st>>>(ctx->pw_kids, ctx->pw_order, ctx->pw_level_off, ctx->pw_nlevel, (int)nl,
                                ctx->pw_vals, out_dev);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

static int upload_spline_table(psc_ctx* ctx, psc_spline_dev** out) {
  std::vector<psc_spline_dev> t(ctx->species.size() * 5);
  for (size_t s = 0; s < ctx->species.size(); ++s)
    for (int f = 0; f < 5; ++f) {
      const psc_species& sp = ctx->species[s];
      t[5 * s + f] = {sp.x[f], sp.z[f], sp.c[f], sp.d[f], sp.nk[f]};
    }
  PSC_CUDA(ctx, psc_dmalloc(out, t.size() * sizeof(psc_spline_dev)));
  PSC_CUDA(ctx, cudaMemcpy(*out, t.data(), t.size() * sizeof(psc_spline_dev), cudaMemcpyHostToDevice));
  return 0;
}

// SAD setup.  Atoms in species-major order; xyz in bohr; h3 = h**3 and
// fourpi = 4*pi as the host computes them.  info (host) receives
// [electron_count_initial, electron_count_normalized].
extern "C" int psc_sad_setup(psc_ctx* ctx, int natoms, const int* species, const double* xyz, double radius,
                             double h3, double fourpi, double z_sum, double* rho0, double* hpot0,
                             double* ppot, double* info, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, natoms >= 1, "sad_setup: no atoms");
  cudaStream_t st = (cudaStream_t)stream;
  for (int a = 0; a < natoms; ++a)
    PSC_REQUIRE(ctx, species[a] >= 0 && species[a] < (int)ctx->species.size() && ctx->species[species[a]].valid,
                "sad_setup: species table missing");
  psc_spline_dev* tab = nullptr;
  if (upload_spline_table(ctx, &tab)) return 1;
  int* sp_d = nullptr;
  double* xyz_d = nullptr;
  PSC_CUDA(ctx, psc_dmalloc(&sp_d, natoms * sizeof(int)));
  PSC_CUDA(ctx, psc_dmalloc(&xyz_d, 3 * natoms * sizeof(double)));
  PSC_CUDA(ctx, cudaMemcpyAsync(sp_d, species, natoms * sizeof(int), cudaMemcpyHostToDevice, st));
  PSC_CUDA(ctx, cudaMemcpyAsync(xyz_d, xyz, 3 * natoms * sizeof(double), cudaMemcpyHostToDevice, st));
  k_sad<<<148 * 8, 256, 0, st>>>(ctx->nx, ctx->ny, ctx->nz, ctx->h, radius, natoms, sp_d, xyz_d, tab, h3, fourpi,
                                 rho0, hpot0, ppot);
  PSC_LAUNCH_CHECK(ctx);
  double* sum_d = ctx->scalars + 200;
  int rc = psc_numpy_sum(ctx, rho0, ctx->n, sum_d, st);
  if (rc) return rc;
  PSC_CUDA(ctx, cudaMemcpyAsync(&ctx->host_scalars[200], sum_d, sizeof(double), cudaMemcpyDeviceToHost, st));
  k_scale_div<<<148 * 8, 256, 0, st>>>(rho0, ctx->n, nullptr, z_sum, sum_d);
  PSC_LAUNCH_CHECK(ctx);
  rc = psc_numpy_sum(ctx, rho0, ctx->n, sum_d + 1, st);
  if (rc) return rc;
  PSC_CUDA(ctx, cudaMemcpyAsync(&ctx->host_scalars[201], sum_d + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  if (info) { info[0] = ctx->host_scalars[200]; info[1] = ctx->host_scalars[201]; }
  psc_dfree(tab); psc_dfree(sp_d); psc_dfree(xyz_d);
  return 0;
}

// ---------------------------------------------------------------------------
// projector geometry
// ---------------------------------------------------------------------------
__global__ void k_nl_box(int nbox, const int* __restrict__ box, const long* __restrict__ start, long total,
                         const double* __restrict__ xyz, const double* __restrict__ rcut_box, double h, double rad,
                         unsigned char* __restrict__ mask) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nbox - 1;
    while (lo < hi) {  // last box whose start <= t
      const int mid = (lo + hi + 1) >> 1;
      if (start[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const int* b = box + 8 * lo;
    const long li = t - start[lo];
    const int ni = b[1] - b[0] + 1, nj = b[3] - b[2] + 1;
    const int ii = b[0] + (int)(li % ni);
    const int jj = b[2] + (int)((li / ni) % nj);
    const int kk = b[4] + (int)(li / ((long)ni * nj));
    const int a = b[6];
    const double xxx = (double)(ii - 1) * h - rad - xyz[3 * a + 0];
    const double yyy = (double)(jj - 1) * h - rad - xyz[3 * a + 1];
    const double zzz = (double)(kk - 1) * h - rad - xyz[3 * a + 2];
    const double dd = sqrt((xxx * xxx + yyy * yyy) + zzz * zzz);
    mask[t] = (dd > 0.0 && dd < rcut_box[lo]) ? 1 : 0;
  }
}

int psc_nl_box_distances(psc_ctx* ctx, int nbox, const int* box_dev, const double* xyz_dev, long total,
                         const long* box_start_dev, double radius, unsigned char* mask_dev, cudaStream_t st) {
  std::vector<int> box(8 * (size_t)nbox);
  PSC_CUDA(ctx, cudaMemcpyAsync(box.data(), box_dev, box.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  std::vector<double> rc(nbox);
  for (int i = 0; i < nbox; ++i) rc[i] = ctx->species[box[8 * i + 7]].rcut;
  double* rc_d = nullptr;
  PSC_CUDA(ctx, psc_dmalloc(&rc_d, nbox * sizeof(double)));
  PSC_CUDA(ctx, cudaMemcpyAsync(rc_d, rc.data(), nbox * sizeof(double), cudaMemcpyHostToDevice, st));
  const int nb = (int)std::max<long>(1, std::min<long>(148L * 8, (total + 255) / 256));
  k_nl_box<<<nb, 256, 0, st>>>(nbox, box_dev, box_start_dev, total, xyz_dev, rc_d, ctx->h, radius, mask_dev);
  PSC_LAUNCH_CHECK(ctx);
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  psc_dfree(rc_d);
  return 0;
}

__global__ void k_nl_u(long npts, const int* __restrict__ idx, const int* __restrict__ pt_atom,
                       const int* __restrict__ atom_sp, const double* __restrict__ xyz,
                       const psc_spline_dev* __restrict__ tab, int nx, int ny, double h, double rad,
                       double* __restrict__ u) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < npts; p += (long)gridDim.x * blockDim.x) {
    const int g = idx[p];
    const int i = g % nx, j = (g / nx) % ny, k = g / (nx * ny);
    const int a = pt_atom[p];
    const double xxx = (double)i * h - rad - xyz[3 * a + 0];
    const double yyy = (double)j * h - rad - xyz[3 * a + 1];
    const double zzz = (double)k * h - rad - xyz[3 * a + 2];
    const double dd = sqrt((xxx * xxx + yyy * yyy) + zzz * zzz);
    const psc_spline_dev* t = tab + 5 * atom_sp[a];
    const double vspp = spline_eval(t[4], dd);
    const double wavpp = spline_eval(t[3], dd);
    u[p] = xxx / dd * wavpp * vspp;
    u[npts + p] = yyy / dd * wavpp * vspp;
    u[2 * npts + p] = zzz / dd * wavpp * vspp;
  }
}

int psc_nl_eval_u(psc_ctx* ctx, long npts, const int* idx_dev, const int* pt_atom_dev, const int* atom_species_dev,
                  const double* xyz_dev, double radius, double* u_dev, cudaStream_t st) {
  psc_spline_dev* tab = nullptr;
  if (upload_spline_table(ctx, &tab)) return 1;
  const int nb = (int)std::max<long>(1, std::min<long>(148L * 8, (npts + 255) / 256));
  k_nl_u<<<nb, 256, 0, st>>>(npts, idx_dev, pt_atom_dev, atom_species_dev, xyz_dev, tab, ctx->nx, ctx->ny, ctx->h,
                             radius, u_dev);
  PSC_LAUNCH_CHECK(ctx);
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  psc_dfree(tab);
  return 0;
}

// ---------------------------------------------------------------------------
// ML density file -> starting charge (V_ion/pseudoDiag_ML4Den_poisson.py:392-530):
//   rho1 = (d * a0^3) * h^3 (d in 1/A^3, flat x-fastest), negatives set to 0,
//   rho1 = Z_sum * rho1 / sum(rho1), hrhs = (4 pi / h^3) (rho1 - rho0);
// sums in NumPy's pairwise order.  info (host, 3): electron count after the
// conversion, number of negative values, electron count after normalisation.
// ---------------------------------------------------------------------------
__global__ void k_ml_scale(const double* __restrict__ raw, double* __restrict__ rho, long n, double a03, double h3) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    rho[i] = (raw[i] * a03) * h3;
}

__global__ void k_ml_clamp(double* __restrict__ rho, long n, unsigned long long* neg) {
  unsigned long long c = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    if (rho[i] < 0.0) { rho[i] = 0.0; ++c; }
  if (c) atomicAdd(neg, c);
}

__global__ void k_ml_norm(double* __restrict__ rho, const double* __restrict__ rho0, double* __restrict__ hrhs, long n,
                          double z_sum, const double* __restrict__ total, double fourpi_h3) {
  const double s = *total;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double v = (z_sum * rho[i]) / s;
    rho[i] = v;
    hrhs[i] = fourpi_h3 * (v - rho0[i]);
  }
}

extern "C" int psc_ml_density(psc_ctx* ctx, const double* raw, double a03, double h3, double z_sum, const double* rho0,
                              double fourpi_h3, double* rho1, double* hrhs, double* info, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, raw && rho0 && rho1 && hrhs && raw != rho1, "ml_density: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const long n = ctx->n;
  const int nb = 148 * 4;
  double* sc = ctx->scalars + 104;  // [0] count after conversion, [1] sum before normalising, [2] count after
  unsigned long long* neg = reinterpret_cast<unsigned long long*>(ctx->scalars + 108);
  PSC_CUDA(ctx, cudaMemsetAsync(neg, 0, sizeof(unsigned long long), st));
  k_ml_scale<<<nb, 256, 0, st>>>(raw, rho1, n, a03, h3);
  PSC_LAUNCH_CHECK(ctx);
  int rc = psc_numpy_sum(ctx, rho1, n, sc + 0, st);
  if (rc) return rc;
  k_ml_clamp<<<nb, 256, 0, st>>>(rho1, n, neg);
  PSC_LAUNCH_CHECK(ctx);
  rc = psc_numpy_sum(ctx, rho1, n, sc + 1, st);
  if (rc) return rc;
  k_ml_norm<<<nb, 256, 0, st>>>(rho1, rho0, hrhs, n, z_sum, sc + 1, fourpi_h3);
  PSC_LAUNCH_CHECK(ctx);
  rc = psc_numpy_sum(ctx, rho1, n, sc + 2, st);
  if (rc) return rc;
  if (info) {
    double h[3];
    unsigned long long negc = 0;
    PSC_CUDA(ctx, cudaMemcpyAsync(h, sc, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    PSC_CUDA(ctx, cudaMemcpyAsync(&negc, neg, sizeof(negc), cudaMemcpyDeviceToHost, st));
    PSC_CUDA(ctx, cudaStreamSynchronize(st));
    info[0] = h[0];
    info[1] = (double)negc;
    info[2] = h[2];
  }
  return 0;
}
