// Internal definitions shared by the libpsc translation units.
//
// libpsc is the device side of the real-space Kohn-Sham SCF hot path:
// matrix-free Hamiltonian H = -0.5*Lap_h + V_nl + diag(pot) on an
// nx*ny*nz cube (x fastest, zero Dirichlet outside), Chebyshev filtering,
// subspace orthonormalisation and Rayleigh-Ritz, Hartree CG, LDA XC,
// multisecant mixing and the SAD/projector setup.  All vectors live in device
// memory owned by the caller; blocks of k vectors are column-major with a
// leading dimension ld.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#define PSC_MAX_DEG 64        // highest Chebyshev degree accepted per filter call
#define PSC_MAX_K 1024        // widest subspace block accepted
#define PSC_RED_BLOCKS 592    // fixed partial-sum count of the deterministic reductions (4 x 148 SMs)
#define PSC_RED_SLOTS 16      // simultaneous dot products per reduction launch
#define PSC_NORM_CHUNKS 32    // row chunks of the column-norm partial sums
#define PSC_WAIT_DEFAULT (1L << 24)  // polls of a bounded device-side wait before it gives up
#define PSC_DRAIN_WAIT (1L << 24)    // polls spent, after a failed wait, on copies and MMAs already issued

enum { PSC_F64 = 0, PSC_F32 = 1 };

struct psc_species {
  // Five natural cubic splines on pruned knots: 0 charge, 1 hartree, 2 pot_S,
  // 3 wfn_P, 4 pot_P - pot_S.  Device arrays x, z, c, d per spline.
  int nk[5] = {0, 0, 0, 0, 0};
  double* x[5] = {nullptr};
  double* z[5] = {nullptr};
  double* c[5] = {nullptr};
  double* d[5] = {nullptr};
  double zvalue = 0.0;  // KB denominator (Zvalue column of the element table)
  double rcut = 0.0;    // projector radius R
  int valid = 0;
};

struct psc_spline_dev {  // flat view handed to kernels
  const double* x;
  const double* z;
  const double* c;
  const double* d;
  int n;
};

struct psc_ctx {
  int device = 0;
  int nx = 0, ny = 0, nz = 0;
  long n = 0;
  double h = 0.0;
  int fd_order = 8;
  int radius = 4;            // stencil half-width (fd_order/2, capped at 4)
  // FP32 stencil weights: 0 plain FP32 weights; 1 plus a correction term for
  // their sum-rule residual in the TMA kernel; 2 that correction folded into
  // the FP32 potential pot32 (calls with another potential, or none, take the
  // term in the kernel)
  int stencil_comp = 2;
  double sumrule32 = 0.0;    // -(c0 + 6 sum_d c_d) of the Hamiltonian weights rounded to FP32, in FP64
  double pot32_shift = 0.0;  // the shift pot32 = fl(pot64 + shift) currently carries
  int stencil_impl = 0;      // 0: TMA pipeline where it applies, 1: register-queue kernel only,
                             // 2: TMA with 2-point FP32 runs, 3 / 4: as 2 / 0 with scalar FP32 arithmetic
  double lap_c0 = 0.0;       // centre weight of A = -Lap_h (1/h^2 folded in)
  double lap_c[4] = {0, 0, 0, 0};
  double ham_c0 = 0.0;       // 0.5 * A weights, as 0.5*(c*(1/(h*h)))
  double ham_c[4] = {0, 0, 0, 0};

  // potential (both precisions)
  double* pot64 = nullptr;
  float* pot32 = nullptr;

  // species tables
  std::vector<psc_species> species;

  // projector tables: n_atoms_nl atoms, compacted ball points
  int nl_atoms = 0;
  long nl_points = 0;
  int* nl_atom_off = nullptr;    // [nl_atoms+1] offsets into the point arrays
  int* nl_idx = nullptr;         // [nl_points] grid index of each ball point
  double* nl_u64 = nullptr;      // [3][nl_points]
  float* nl_u32 = nullptr;       // [3][nl_points]
  double* nl_w = nullptr;        // [nl_atoms] 1/xint = h^3 / Zvalue
  long nl_touched = 0;           // unique grid points covered by any ball
  int* nl_t_idx = nullptr;       // [nl_touched] grid index
  int* nl_t_off = nullptr;       // [nl_touched+1] offsets into nl_t_ent
  int* nl_t_ent = nullptr;       // [nl_points] ball-point ids (atom order)
  int* nl_point_atom = nullptr;  // [nl_points] owning atom of each ball point
  void* nl_proj = nullptr;       // [nl_atoms][3][k] projections (double; reused for float)
  size_t nl_proj_bytes = 0;

  // Chebyshev per-step coefficients (alpha, beta, gamma) on the device
  double* cheb_coef = nullptr;   // [PSC_MAX_DEG+1][3]

  // deterministic reductions
  double* red_partial = nullptr;  // [PSC_RED_SLOTS][PSC_RED_BLOCKS]
  double* scalars = nullptr;      // general device scalar scratch [256]
  double* host_scalars = nullptr; // pinned host mirror [256]

  // small dense work (k x k)
  int dense_cap = 0;
  double* gram = nullptr;        // [cap*cap]
  double* gram2 = nullptr;       // [cap*cap]
  double* evec = nullptr;        // [cap*cap]
  double* tri = nullptr;         // [cap*cap]
  double* eig_work = nullptr;    // [2 (cap+2)^2] eigensolver scratch: reflectors, eigenvectors of T, T, tau
  double* gram_partial = nullptr;// [gram_blocks][cap*cap] Gram partial sums
  int gram_blocks = 0;
  int* dev_status = nullptr;     // device-side error flags [8]
  // tensor-core Gram pair (mixed precision)
  int gram_tc = 1;               // 1: FP32 Gram pairs on tcgen05 (3xTF32), 0: CUDA cores
  long gram_chunk = 0;           // rows per tensor-core Gram chunk (0: four waves of CTAs)
  int* dm_pairs = nullptr;       // upper-triangle tile pairs of the DMMA Gram pair (int2)
  int dm_pairs_cap = 0, dm_pairs_k = -1;
  float* tc_part = nullptr;      // per-chunk FP32 partial tiles
  size_t tc_part_floats = 0;
  void* tc_pairs = nullptr;      // int2 tile pairs (upper triangle)
  int tc_pairs_k = 0;
  // tensor-core block product W T (mixed precision Rayleigh-Ritz)
  int gemm_tc = 1;               // 1: FP32 W T on tcgen05 (3xTF32), 0: CUDA cores
  float* tsplit = nullptr;       // T split into TF32 hi/lo B tiles
  size_t tsplit_floats = 0;
  double* dens_w = nullptr;      // [1024] density weight per state (k_density_weights)
  // NumPy-order pairwise sum: leaf ranges and the tree above them for length pw_n
  long pw_n = 0;
  void* pw_buf = nullptr;
  long* pw_lo = nullptr;
  long* pw_len = nullptr;
  double* pw_vals = nullptr;
  int2* pw_kids = nullptr;
  int* pw_order = nullptr;
  int* pw_level_off = nullptr;
  long pw_nleaf = 0;
  int pw_nlevel = 0;
  // learned-start convolution forward: 2 tcgen05 implicit GEMM, 0 CUDA cores,
  // 1 by layer (tcgen05 from 32 output channels)
  int conv_tc = 1;
  void* conv_wt = nullptr;       // BF16 weights transposed to [Cout rounded to 16][K rounded to 64]
  size_t conv_wt_bytes = 0;
  // sphere mask of the Hamiltonian (0: the whole cube): H X is zero at
  // points farther than sqrt(mask_r2) from mask_c (the cube's centre)
  double mask_r2 = 0.0;
  double mask_c[3] = {0.0, 0.0, 0.0};
  // polls of every bounded device-side wait before it gives up (status words 3-7)
  long wait_limit = PSC_WAIT_DEFAULT;
  // exact squared column norms of FP32 blocks (density normalisation)
  double* col_norm_part = nullptr;  // [cap][PSC_NORM_CHUNKS]
  int col_norm_cap = 0;

  // TMA stencil work tables (column, slab, z range per CTA), one per launch shape
  struct StencilSched {
    long long key = 0;
    int n = 0;
    int* dev = nullptr;
    std::vector<int> host;   // the uploaded copy (kept alive for the asynchronous upload)
  };
  std::vector<StencilSched> st_sched;

  // spectral Poisson preconditioner: DST-I matrices (m x mp, mp = m rounded
  // up to 16), per-axis eigenvalues of the stencil, two work vectors
  double* spec_S[3] = {nullptr, nullptr, nullptr};
  double* spec_lam[3] = {nullptr, nullptr, nullptr};
  int spec_mp[3] = {0, 0, 0};
  double* spec_tmp = nullptr;

  // Lanczos vectors (double)
  double* lz_v = nullptr;        // [3][n]
  double* lz_basis = nullptr;    // [7][n] basis of the six-step bound of chefsi1
  // tridiagonal eigensolver: LU factors of T - lambda I per cluster start
  double* tri_work = nullptr;
  size_t tri_work_doubles = 0;

  // PCG vectors (double)
  double* cg_r = nullptr;
  double* cg_p = nullptr;
  double* cg_ap = nullptr;
  double* cg_part = nullptr;     // [2][cg_part_cap] per-CTA partial sums
  int cg_part_cap = 0;
  double* cg_x = nullptr;        // solution buffer the captured CG graph works on
  double* cg_p2 = nullptr;       // second direction buffer (the two alternate)
  double* cg_ro = nullptr;       // r.r before each iteration
  unsigned int* cg_bar = nullptr;  // grid-barrier arrival counter of the persistent CG
  int cg_persistent = 1;         // 1: persistent cooperative CG when the vectors fit in shared memory
  cudaGraphExec_t cg_exec = nullptr;
  cudaStream_t cap_stream = nullptr;  // private stream used only for graph capture
  int use_graphs = 1;

  // mixer history
  int mix_cap = 0;
  int mix_m = 0;                 // columns in DX/DF
  double* mix_dx = nullptr;      // [cap][n]
  double* mix_df = nullptr;      // [cap][n]
  double* mix_nv = nullptr;      // [n]  (group vector N for group size 1)
  double* mix_tmp = nullptr;     // [n]
  double* mix_coef = nullptr;    // [3*cap + 8] dot products and scalars
  double* mix_partial = nullptr; // [3*cap + 2][PSC_RED_BLOCKS]
  double mix_last_fnorm = -1.0;

  std::string last_error;
};

// ---------------------------------------------------------------------------
// device memory
// ---------------------------------------------------------------------------
// Context memory comes from CUDA's stream-ordered pool (legacy default
// stream), whose release threshold is raised once per device so that freed
// blocks stay in the pool: a process that runs many SCFs pays the cost of
// mapping fresh device memory once, not at every context creation.
cudaError_t psc_dmalloc_bytes(void** p, size_t bytes);
void psc_dfree(void* p);
template <typename T>
inline cudaError_t psc_dmalloc(T** p, size_t bytes) {
  return psc_dmalloc_bytes(reinterpret_cast<void**>(p), bytes);
}

// ---------------------------------------------------------------------------
// error plumbing
// ---------------------------------------------------------------------------
void psc_set_error(psc_ctx* ctx, const std::string& msg);

#define PSC_CUDA(ctx, call)                                                            \
  do {                                                                                 \
    cudaError_t _e = (call);                                                           \
    if (_e != cudaSuccess) {                                                           \
      psc_set_error((ctx), std::string(#call) + ": " + cudaGetErrorString(_e));        \
      return 1;                                                                        \
    }                                                                                  \
  } while (0)

// Every kernel launch site is followed by exactly one PSC_LAUNCH_CHECK, which
// also counts the launch (psc_launch_count).
void psc_note_launch();
#define PSC_LAUNCH_CHECK(ctx)                                                          \
  do {                                                                                 \
    psc_note_launch();                                                                 \
    cudaError_t _e = cudaGetLastError();                                               \
    if (_e != cudaSuccess) {                                                           \
      psc_set_error((ctx), std::string("kernel launch: ") + cudaGetErrorString(_e) +   \
                               " at " + __FILE__ + ":" + std::to_string(__LINE__));    \
      return 1;                                                                        \
    }                                                                                  \
  } while (0)

#define PSC_REQUIRE(ctx, cond, msg)                                                    \
  do {                                                                                 \
    if (!(cond)) {                                                                     \
      psc_set_error((ctx), std::string(msg));                                          \
      return 2;                                                                        \
    }                                                                                  \
  } while (0)

static inline int psc_div_up(long a, long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T psc_warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of one value per thread; result valid in thread 0.  The
// combine order is fixed, so the result is reproducible run to run.
template <typename T, int NT>
__device__ __forceinline__ T psc_block_sum(T v, T* sh /* >= NT/32 */) {
  v = psc_warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  T r = T(0);
  if (w == 0) {
    r = (l < NT / 32) ? sh[l] : T(0);
    r = psc_warp_sum(r);
  }
  return r;
}

// Ceperley-Alder / Perdew-Zunger LDA of one density value r (electrons per
// bohr^3), V_xc/exc_nspn.py:73-91: returns v_xc (Ry) and adds the point's
// energy density 0.75 r v_x + r eps_c to e.  Points with r <= 0 give 0.
// Shared by k_xc (scf.cu) and k_xc_noalloc (noalloc.cu).
__device__ __forceinline__ double psc_lda_point(double r, double& e) {
  const double g = -0.2846, b1 = 1.0529, b2 = 0.3334;
  const double c1 = 0.0622, c2 = 0.096, c3 = 0.004, c4 = 0.0232, c5 = 0.0192;
  const double third = 1.0 / 3.0;
  const double pi = 3.141592653589793;
  const double a0 = pow(4.0 / (9.0 * pi), third);
  const double twovpia0 = 2.0 / (pi * a0);
  const double p75vpi = 0.75 / pi;
  double v = 0.0;
  if (r > 0.0) {
    const double rs = pow(p75vpi / r, third);
    v = -twovpia0 / rs;
    double ec;
    e += 0.75 * r * v;
    if (rs >= 1.0) {
      const double sq = sqrt(rs);
      ec = g / (1.0 + b1 * sq + b2 * rs);
      v += (ec * ec) * (1.0 + 3.5 * b1 * sq * third + 4.0 * b2 * rs * third) / g;
    } else {
      const double al = log(rs);
      ec = c1 * al - c2 + (c3 * al - c4) * rs;
      v += ec - (c1 + (c3 * al - c5) * rs) * third;
    }
    e += r * ec;
  }
  return v;
}

// max / min that propagate NaN, as numpy.max / numpy.min do (fmax / fmin
// would drop it)
__device__ __forceinline__ double psc_nanmax(double a, double b) { return (a != a || b != b) ? a + b : fmax(a, b); }
__device__ __forceinline__ double psc_nanmin(double a, double b) { return (a != a || b != b) ? a + b : fmin(a, b); }

// ---------------------------------------------------------------------------
// cross-unit host entry points used internally
// ---------------------------------------------------------------------------
// Deterministic multi-dot: out[s] = sum_i a_s[i]*b_s[i] for s < nslots (device result).
int psc_dots(psc_ctx* ctx, int nslots, const double* const* a, const double* const* b, long n,
             double* out_dev, cudaStream_t st);
int psc_ensure_dense(psc_ctx* ctx, int k);
int psc_ensure_proj(psc_ctx* ctx, int k);
int psc_apply_h_impl(psc_ctx* ctx, int dtype, const void* X, long ldx, void* Y, long ldy,
                     const void* P, long ldp, int k, const double* coef_dev, double a, double b,
                     double g, cudaStream_t st);
int psc_gram_impl(psc_ctx* ctx, int dtype, const void* A, long lda, const void* B, long ldb, int k,
                  double* out, int symmetrize, cudaStream_t st);
int psc_gemm_nn_impl(psc_ctx* ctx, int dtype, const void* W, long ldw, int k, const double* Q,
                     int kout, void* out, long ldo, cudaStream_t st);
int psc_syev_impl(psc_ctx* ctx, double* A, int k, double* evals, double* evecs, cudaStream_t st);
int psc_tridiag_eig_impl(psc_ctx* ctx, const double* ab, int k, int nvec, double* evals, double* Z, long ldz,
                         double crel, cudaStream_t st);
int psc_stencil_blocks(psc_ctx* ctx, int k);
int psc_laplacian_fused(psc_ctx* ctx, const double* x, const double* prev, double* y, double a, double b,
                        double g, double* dot_partial, int* nblocks, cudaStream_t st);
int psc_random_impl(psc_ctx* ctx, int dtype, int dist, unsigned long long seed, void* out, long ld,
                    long rows, int cols, cudaStream_t st);
// zero the points outside the sphere mask in k columns (no-op without a mask)
int psc_mask_block_impl(psc_ctx* ctx, int dtype, void* X, long ld, int k, cudaStream_t st);
// FP32 block product W T on tensor cores; -1 when it does not apply
int psc_gram_pair_dmma(psc_ctx* ctx, int dtype, const void* W, const void* V, long ld, int k, double* S, double* K,
                       cudaStream_t st);
int psc_gemm_tall_dmma(psc_ctx* ctx, int dtype, const void* W, long ldw, int k, const double* Tm, int kout, void* O,
                       long ldo, cudaStream_t st);
int psc_gemm_tall_tc(psc_ctx* ctx, const float* W, long ld, int k, const double* Tm, int kout, float* O, long ldo,
                     cudaStream_t st);
// FP32 Gram pair on tensor cores; -1 when it does not apply
int psc_gram_pair_tc(psc_ctx* ctx, const float* W, const float* V, long ld, int k, double* S, double* K,
                     cudaStream_t st);
