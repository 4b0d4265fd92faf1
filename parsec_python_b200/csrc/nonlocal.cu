// Kleinman-Bylander nonlocal term in factored form and its setup.
//
// V_nl = sum_a sum_m u_am u_am^T / xint_a  (V_ion/pseudoNL_original.py:187-206)
// is applied as  Y[idx] += alpha * sum_a sum_m u_am * (w_a * u_am . X[idx]),
// w_a = 1/xint_a = h^3 / Zvalue_a, never forming the n_a x n_a blocks.
//   project: one warp per (atom, column) reduces w_a * U_a^T X (3 values)
//            over the ball with a fixed shuffle tree;
//   scatter: one thread per (touched grid point, group of 8 columns) adds
//            the sum over the balls covering that point, in atom order.  No
//            atomics, so the result is bitwise reproducible.
#include "psc_internal.cuh"
#include "../../include/psc.h"

#include <algorithm>
#include <cmath>
#include <numeric>

// Projection: one CTA per (atom, group of NL_KC columns), one warp per
// column.  The ball's grid indices and u values are staged in shared memory
// NL_STAGE points at a time; lane l of a warp takes points l, l + 32, ...
// (NL_UNROLL gathers in flight), then a fixed shuffle tree sums the lanes,
// so the result is reproducible.  Many warps per SM keep enough gathers in
// flight for HBM, which a few threads per ball point could not.
constexpr int NL_KC = 16;       // columns (warps) per projection CTA
constexpr int NL_STAGE = 1024;  // ball points staged per pass
constexpr int NL_UNROLL = 4;

template <typename T>
__global__ void __launch_bounds__(NL_KC * 32)
k_nl_project(const T* __restrict__ X, long ldx, int k, const int* __restrict__ atom_off,
             const int* __restrict__ idx, const T* __restrict__ u, long npts, const double* __restrict__ w,
             double* __restrict__ proj) {
  __shared__ int s_idx[NL_STAGE];
  __shared__ T s_u[3][NL_STAGE];
  const int a = blockIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int c = blockIdx.y * NL_KC + wid;
  const int lo = atom_off[a], hi = atom_off[a + 1];
  const T* Xc = X + (long)min(c, k - 1) * ldx;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int b = lo; b < hi; b += NL_STAGE) {
    const int nb = min(NL_STAGE, hi - b);
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += NL_KC * 32) {
      s_idx[i] = idx[b + i];
      s_u[0][i] = u[b + i];
      s_u[1][i] = u[npts + b + i];
      s_u[2][i] = u[2 * npts + b + i];
    }
    __syncthreads();
    for (int i0 = lane; i0 < nb; i0 += 32 * NL_UNROLL) {
      double xv[NL_UNROLL];
#pragma unroll
      for (int r = 0; r < NL_UNROLL; ++r) {
        const int i = i0 + 32 * r;
        xv[r] = i < nb ? (double)Xc[s_idx[i]] : 0.0;
      }
#pragma unroll
      for (int r = 0; r < NL_UNROLL; ++r) {
        const int i = i0 + 32 * r;
        if (i < nb) {
          s0 += (double)s_u[0][i] * xv[r];
          s1 += (double)s_u[1][i] * xv[r];
          s2 += (double)s_u[2][i] * xv[r];
        }
      }
    }
  }
  s0 = psc_warp_sum(s0);
  s1 = psc_warp_sum(s1);
  s2 = psc_warp_sum(s2);
  if (lane == 0 && c < k) {
    const double wa = w[a];
    proj[((long)a * 3 + 0) * k + c] = wa * s0;
    proj[((long)a * 3 + 1) * k + c] = wa * s1;
    proj[((long)a * 3 + 2) * k + c] = wa * s2;
  }
}

// Scatter: one thread per (touched grid point, group of NL_SC columns); the
// entries covering the point and their u values are read once for every
// column of the group, the group's Y values are loaded before the sums and
// stored after them, and each column's sum runs over the entries in atom
// order (no atomics, so the result is bitwise reproducible).
constexpr int NL_SC = 8;
template <typename T>
__global__ void __launch_bounds__(256)
k_nl_scatter(T* __restrict__ Y, long ldy, int k, long ntouched, const int* __restrict__ t_idx,
             const int* __restrict__ t_off, const int* __restrict__ t_ent, const int* __restrict__ pt_atom,
             const T* __restrict__ u, long npts, const double* __restrict__ proj, const double* __restrict__ coef,
             double ha) {
  const int ngrp = (k + NL_SC - 1) / NL_SC;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= ntouched * (long)ngrp) return;
  const double alpha = coef ? coef[0] : ha;
  const long pt = t % ntouched;
  const int c0 = (int)(t / ntouched) * NL_SC;
  const int nc = min(NL_SC, k - c0);
  T* yp = Y + (long)t_idx[pt] + (long)c0 * ldy;
  T yv[NL_SC];
#pragma unroll
  for (int c = 0; c < NL_SC; ++c) yv[c] = c < nc ? yp[(long)c * ldy] : T(0);
  double s[NL_SC];
#pragma unroll
  for (int c = 0; c < NL_SC; ++c) s[c] = 0.0;
  for (int e = t_off[pt]; e < t_off[pt + 1]; ++e) {
    const int p = t_ent[e];
    const double u0 = (double)u[p], u1 = (double)u[npts + p], u2 = (double)u[2 * npts + p];
    const double* pr = proj + (long)pt_atom[p] * 3 * k + c0;
#pragma unroll
    for (int c = 0; c < NL_SC; ++c)
      if (c < nc) s[c] += u0 * pr[c] + u1 * pr[k + c] + u2 * pr[2 * k + c];
  }
#pragma unroll
  for (int c = 0; c < NL_SC; ++c)
    if (c < nc) yp[(long)c * ldy] = (T)((double)yv[c] + alpha * s[c]);
}

int psc_ensure_proj(psc_ctx* ctx, int k) {
  size_t need = (size_t)std::max(ctx->nl_atoms, 1) * 3 * k * sizeof(double);
  if (need > ctx->nl_proj_bytes) {
    psc_dfree(ctx->nl_proj);
    ctx->nl_proj = nullptr;
    PSC_CUDA(ctx, psc_dmalloc(&ctx->nl_proj, need));
    ctx->nl_proj_bytes = need;
  }
  return 0;
}

int psc_nl_project(psc_ctx* ctx, int dtype, const void* X, long ldx, int k, cudaStream_t st) {
  if (psc_ensure_proj(ctx, k)) return 1;
  dim3 grid(ctx->nl_atoms, (k + NL_KC - 1) / NL_KC);
  if (dtype == PSC_F64)
    k_nl_project<double><<<grid, NL_KC * 32, 0, st>>>((const double*)X, ldx, k, ctx->nl_atom_off, ctx->nl_idx,
                                                       ctx->nl_u64, ctx->nl_points, ctx->nl_w,
                                                       (double*)ctx->nl_proj);
  else
    k_nl_project<float><<<grid, NL_KC * 32, 0, st>>>((const float*)X, ldx, k, ctx->nl_atom_off, ctx->nl_idx,
                                                      ctx->nl_u32, ctx->nl_points, ctx->nl_w,
                                                      (double*)ctx->nl_proj);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

int psc_nl_scatter(psc_ctx* ctx, int dtype, void* Y, long ldy, int k, const double* coef, double a,
                   cudaStream_t st) {
  const long total = ctx->nl_touched * (long)((k + NL_SC - 1) / NL_SC);
  if (total == 0) return 0;
  PSC_REQUIRE(ctx, (total + 255) / 256 <= INT32_MAX, "nl_scatter: too many touched points x columns");
  const int nb = (int)((total + 255) / 256);   // one (touched point, column group) per thread
  if (dtype == PSC_F64)
    k_nl_scatter<double><<<nb, 256, 0, st>>>((double*)Y, ldy, k, ctx->nl_touched, ctx->nl_t_idx,
                                              ctx->nl_t_off, ctx->nl_t_ent, ctx->nl_point_atom, ctx->nl_u64,
                                              ctx->nl_points, (const double*)ctx->nl_proj, coef, a);
  else
    k_nl_scatter<float><<<nb, 256, 0, st>>>((float*)Y, ldy, k, ctx->nl_touched, ctx->nl_t_idx, ctx->nl_t_off,
                                             ctx->nl_t_ent, ctx->nl_point_atom, ctx->nl_u32, ctx->nl_points,
                                             (const double*)ctx->nl_proj, coef, a);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

void psc_free_projectors(psc_ctx* ctx) {
  psc_dfree(ctx->nl_atom_off); psc_dfree(ctx->nl_idx); psc_dfree(ctx->nl_u64); psc_dfree(ctx->nl_u32);
  psc_dfree(ctx->nl_w); psc_dfree(ctx->nl_t_idx); psc_dfree(ctx->nl_t_off); psc_dfree(ctx->nl_t_ent);
  psc_dfree(ctx->nl_point_atom); psc_dfree(ctx->nl_proj);
  ctx->nl_atom_off = ctx->nl_idx = ctx->nl_t_idx = ctx->nl_t_off = ctx->nl_t_ent = ctx->nl_point_atom = nullptr;
  ctx->nl_u64 = nullptr; ctx->nl_u32 = nullptr; ctx->nl_w = nullptr; ctx->nl_proj = nullptr;
  ctx->nl_proj_bytes = 0;
  ctx->nl_atoms = 0; ctx->nl_points = 0; ctx->nl_touched = 0;
}

int psc_nl_apply_mask(psc_ctx* ctx, cudaStream_t st);


// setup.cu
int psc_nl_box_distances(psc_ctx* ctx, int nbox, const int* box_dev /* [nbox][8] */, const double* xyz_dev,
                         long total, const long* box_start_dev, double radius, unsigned char* mask_dev,
                         cudaStream_t st);
int psc_nl_eval_u(psc_ctx* ctx, long npts, const int* idx_dev, const int* pt_atom_dev,
                  const int* atom_species_dev, const double* xyz_dev, double radius, double* u_dev,
                  cudaStream_t st);

// Build the projector tables for the atoms (species ids and coordinates in
// bohr, species-major order as in pseudoNL_original.py:60-115).
extern "C" int psc_projector_setup(psc_ctx* ctx, int natoms, const int* species, const double* xyz,
                                   double radius, void* stream) {
  if (!ctx) return 2;
  PSC_REQUIRE(ctx, natoms >= 0, "projector_setup: natoms < 0");
  cudaStream_t st = (cudaStream_t)stream;
  psc_free_projectors(ctx);
  if (natoms == 0) return 0;
  const double h = ctx->h;
  const int nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
  // per-atom window boxes (1-based inclusive ranges), pseudoNL_original.py:122-138
  std::vector<int> box;          // [imin, imax, jmin, jmax, kmin, kmax, atom, species]
  std::vector<long> start;
  long total = 0;
  for (int a = 0; a < natoms; ++a) {
    const int sp = species[a];
    PSC_REQUIRE(ctx, sp >= 0 && sp < (int)ctx->species.size() && ctx->species[sp].valid,
                "projector_setup: species table missing");
    const double R = ctx->species[sp].rcut;
    const double xa = xyz[3 * a], ya = xyz[3 * a + 1], za = xyz[3 * a + 2];
    // Python round() is round-half-even, as is nearbyint in the default mode.
    const int i0 = (int)std::nearbyint((xa + radius) / h + 1);
    const int j0 = (int)std::nearbyint((ya + radius) / h + 1);
    const int k0 = (int)std::nearbyint((za + radius) / h + 1);
    const int span = (int)std::nearbyint(R / h);
    int b[8] = {std::max(1, i0 - span), std::min(nx, i0 + span), std::max(1, j0 - span),
                std::min(ny, j0 + span), std::max(1, k0 - span), std::min(nz, k0 + span), a, sp};
    if (b[0] > b[1] || b[2] > b[3] || b[4] > b[5]) continue;
    box.insert(box.end(), b, b + 8);
    start.push_back(total);
    total += (long)(b[1] - b[0] + 1) * (b[3] - b[2] + 1) * (b[5] - b[4] + 1);
  }
  const int nbox = (int)start.size();
  if (nbox == 0) return 0;
  std::vector<double> xyzv(xyz, xyz + 3 * (long)natoms);
  std::vector<int> atom_species(species, species + natoms);
  int *box_d = nullptr, *asp_d = nullptr;
  long* start_d = nullptr;
  double* xyz_d = nullptr;
  unsigned char* mask_d = nullptr;
  auto cleanup = [&]() { psc_dfree(box_d); psc_dfree(start_d); psc_dfree(xyz_d); psc_dfree(mask_d); psc_dfree(asp_d); };
  PSC_CUDA(ctx, psc_dmalloc(&box_d, box.size() * sizeof(int)));
  PSC_CUDA(ctx, psc_dmalloc(&start_d, start.size() * sizeof(long)));
  PSC_CUDA(ctx, psc_dmalloc(&xyz_d, xyzv.size() * sizeof(double)));
  PSC_CUDA(ctx, psc_dmalloc(&asp_d, atom_species.size() * sizeof(int)));
  PSC_CUDA(ctx, psc_dmalloc(&mask_d, total));
  PSC_CUDA(ctx, cudaMemcpyAsync(box_d, box.data(), box.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  PSC_CUDA(ctx, cudaMemcpyAsync(start_d, start.data(), start.size() * sizeof(long), cudaMemcpyHostToDevice, st));
  PSC_CUDA(ctx, cudaMemcpyAsync(xyz_d, xyzv.data(), xyzv.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  PSC_CUDA(ctx, cudaMemcpyAsync(asp_d, atom_species.data(), atom_species.size() * sizeof(int),
                                cudaMemcpyHostToDevice, st));
  if (psc_nl_box_distances(ctx, nbox, box_d, xyz_d, total, start_d, radius, mask_d, st)) { cleanup(); return 1; }
  std::vector<unsigned char> mask(total);
  PSC_CUDA(ctx, cudaMemcpyAsync(mask.data(), mask_d, total, cudaMemcpyDeviceToHost, st));
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  // Compact in window order (k, j, i loops) per atom; record grid index and owner.
  std::vector<int> atom_off{0}, idx, pt_atom, nl_atom_of_box;
  for (int bi = 0; bi < nbox; ++bi) {
    const int* b = &box[8 * bi];
    long t = start[bi];
    int cnt = 0;
    for (int kk = b[4]; kk <= b[5]; ++kk)
      for (int jj = b[2]; jj <= b[3]; ++jj)
        for (int ii = b[0]; ii <= b[1]; ++ii, ++t)
          if (mask[t]) {
            idx.push_back((ii - 1) + nx * ((jj - 1) + (kk - 1) * ny));
            pt_atom.push_back((int)nl_atom_of_box.size());
            ++cnt;
          }
    if (cnt == 0) continue;
    nl_atom_of_box.push_back(b[6]);
    atom_off.push_back((int)idx.size());
  }
  const int nla = (int)nl_atom_of_box.size();
  const long npts = (long)idx.size();
  psc_dfree(mask_d); mask_d = nullptr;
  if (nla == 0) { cleanup(); return 0; }
  // touched points: entries sorted by grid index, ties in atom order
  std::vector<int> order(npts);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return idx[x] < idx[y]; });
  std::vector<int> t_idx, t_off{0}, t_ent;
  for (long i = 0; i < npts; ++i) {
    const int p = order[i];
    if (t_idx.empty() || t_idx.back() != idx[p]) {
      if (!t_idx.empty()) t_off.push_back((int)t_ent.size());
      t_idx.push_back(idx[p]);
    }
    t_ent.push_back(p);
  }
  t_off.push_back((int)t_ent.size());
  std::vector<double> w(nla);
  std::vector<int> nl_sp(nla);
  for (int a = 0; a < nla; ++a) {
    const int at = nl_atom_of_box[a];
    nl_sp[a] = species[at];
    w[a] = 1.0 / (ctx->species[species[at]].zvalue / (h * h * h));
  }
  // per ball point: original atom index for coordinates/species lookup
  std::vector<int> pt_orig(npts);
  for (long p = 0; p < npts; ++p) pt_orig[p] = nl_atom_of_box[pt_atom[p]];
  ctx->nl_atoms = nla;
  ctx->nl_points = npts;
  ctx->nl_touched = (long)t_idx.size();
  PSC_CUDA(ctx, psc_dmalloc(&ctx->nl_atom_off, atom_off.size() * sizeof(int)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->nl_idx, npts * sizeof(int)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->nl_point_atom, npts * sizeof(int)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->nl_u64, 3 * npts * sizeof(double)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->nl_u32, 3 * npts * sizeof(float)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->nl_w, nla * sizeof(double)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->nl_t_idx, t_idx.size() * sizeof(int)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->nl_t_off, t_off.size() * sizeof(int)));
  PSC_CUDA(ctx, psc_dmalloc(&ctx->nl_t_ent, t_ent.size() * sizeof(int)));
  int* pt_orig_d = nullptr;
  PSC_CUDA(ctx, psc_dmalloc(&pt_orig_d, npts * sizeof(int)));
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->nl_atom_off, atom_off.data(), atom_off.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->nl_idx, idx.data(), npts * sizeof(int), cudaMemcpyHostToDevice, st));
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->nl_point_atom, pt_atom.data(), npts * sizeof(int), cudaMemcpyHostToDevice, st));
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->nl_w, w.data(), nla * sizeof(double), cudaMemcpyHostToDevice, st));
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->nl_t_idx, t_idx.data(), t_idx.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->nl_t_off, t_off.data(), t_off.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  PSC_CUDA(ctx, cudaMemcpyAsync(ctx->nl_t_ent, t_ent.data(), t_ent.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  PSC_CUDA(ctx, cudaMemcpyAsync(pt_orig_d, pt_orig.data(), npts * sizeof(int), cudaMemcpyHostToDevice, st));
  int rc = psc_nl_eval_u(ctx, npts, ctx->nl_idx, pt_orig_d, asp_d, xyz_d, radius, ctx->nl_u64, st);
  if (!rc) rc = psc_cast(ctx, PSC_F32, ctx->nl_u64, ctx->nl_u32, 3 * npts, st);
  if (!rc) rc = psc_nl_apply_mask(ctx, st);
  PSC_CUDA(ctx, cudaStreamSynchronize(st));
  psc_dfree(pt_orig_d);
  cleanup();
  return rc;
}

// Sphere mask: the projector functions vanish at ball points outside the
// sphere (their rows and columns of V_nl are those of masked points).
__global__ void k_nl_mask(double* u64, float* u32, const int* __restrict__ idx, long npts, int nx, int ny, double h,
                          double cx, double cy, double cz, double r2) {
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < npts; p += (long)gridDim.x * blockDim.x) {
    const long g = idx[p];
    const double x = (g % nx) * h - cx, y = ((g / nx) % ny) * h - cy, z = (g / ((long)nx * ny)) * h - cz;
    if (x * x + y * y + z * z > r2)
      for (int m = 0; m < 3; ++m) {
        u64[m * npts + p] = 0.0;
        u32[m * npts + p] = 0.0f;
      }
  }
}

int psc_nl_apply_mask(psc_ctx* ctx, cudaStream_t st) {
  if (ctx->mask_r2 <= 0.0 || ctx->nl_points == 0) return 0;
  const long npts = ctx->nl_points;
  k_nl_mask<<<(int)std::min<long>(148L * 8, (npts + 255) / 256), 256, 0, st>>>(
      ctx->nl_u64, ctx->nl_u32, ctx->nl_idx, npts, ctx->nx, ctx->ny, ctx->h, ctx->mask_c[0], ctx->mask_c[1],
      ctx->mask_c[2], ctx->mask_r2);
  PSC_LAUNCH_CHECK(ctx);
  return 0;
}

// Copy the projector tables out (for checks against the reference's V_nl).
extern "C" int psc_projector_export(psc_ctx* ctx, int* atom_off, int* idx, double* u, double* w) {
  if (!ctx) return 2;
  if (ctx->nl_atoms == 0) return 0;
  if (atom_off) PSC_CUDA(ctx, cudaMemcpy(atom_off, ctx->nl_atom_off, (ctx->nl_atoms + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  if (idx) PSC_CUDA(ctx, cudaMemcpy(idx, ctx->nl_idx, ctx->nl_points * sizeof(int), cudaMemcpyDeviceToHost));
  if (u) PSC_CUDA(ctx, cudaMemcpy(u, ctx->nl_u64, 3 * ctx->nl_points * sizeof(double), cudaMemcpyDeviceToHost));
  if (w) PSC_CUDA(ctx, cudaMemcpy(w, ctx->nl_w, ctx->nl_atoms * sizeof(double), cudaMemcpyDeviceToHost));
  return 0;
}
