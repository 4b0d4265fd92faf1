/*
 * libpsc -- C ABI of the B200 (sm_100a) real-space Kohn-Sham SCF hot path.
 *
 * Plain pointers and sizes only.  Vectors are device pointers; a block of k
 * vectors is column-major with leading dimension ld >= n = nx*ny*nz, grid
 * index p = i + nx*(j + ny*k) (x fastest), zero Dirichlet values outside the
 * cube.  `stream` is a cudaStream_t passed as void*.  Every function returns
 * 0 on success, 2 for an invalid argument and 1 for a CUDA error; the message
 * is available from psc_last_error().  Units follow the reference: bohr,
 * Hartree for the Hamiltonian, Rydberg for XC potentials and energies.
 *
 * Each declaration names the part of PARSEC.py (zeyizhang-berkeley/
 * parsec_python, src/) whose behaviour it reproduces.  In the reference these
 * steps sit behind rsdft_backend.select_solver_backend (rsdft_backend.py:80)
 * and the SolverBackend bundle (rsdft_models.py:179-217); XC, mixing and the
 * Laplacian are direct imports in rsdft_solver.py:20-26.
 */
#ifndef PSC_H
#define PSC_H

#ifdef __cplusplus
extern "C" {
#endif

#define PSC_ABI_VERSION 1

typedef struct psc_ctx psc_ctx;

/* element types of vector blocks */
#define PSC_DTYPE_F64 0
#define PSC_DTYPE_F32 1

int psc_version(void);
/* Number of kernels this library has launched in the process so far. */
long long psc_launch_count(void);
const char* psc_last_error(const psc_ctx* ctx);

/* Grid context: nx*ny*nz cube, spacing h (bohr), finite-difference order
 * (orders <= 2, <= 4, <= 6, else 8 as Laplacian/fd3d.py:49-94).
 * Replaces the construction A = (1/h^2) fd3d(...) at rsdft_solver.py:186. */
int psc_ctx_create(int nx, int ny, int nz, double h, int fd_order, psc_ctx** out);
int psc_ctx_destroy(psc_ctx* ctx);
/* out[8] = nx, ny, nz, n, projector atoms, projector points, touched points, stencil radius */
int psc_ctx_info(const psc_ctx* ctx, long* out);
/* host flags[8] of device-side checks: [0] filter bounds inverted, [1]
 * Cholesky pivot <= 0 at column flags[1]-1, [3] TMA stencil wait timed out,
 * [4] persistent CG grid barrier timed out, [5] tensor-core Gram pipeline
 * wait timed out, [6] tensor-core block product pipeline wait timed out,
 * [7] tensor-core convolution pipeline wait timed out; [2] reserved.
 * clear != 0 resets */
int psc_status(psc_ctx* ctx, int* host_flags, int clear, void* stream);
/* Polls of every bounded device-side wait (status words 3-7) before the CTA
 * gives up, records its status word and returns; polls < 0 restores the
 * default (2^24; the CG grid barrier waits 4x as long).  0 makes every wait
 * run out at once (failure-path tests).  No counterpart in the reference. */
int psc_set_wait_limit(psc_ctx* ctx, long polls);

/* ---- ionic setup ------------------------------------------------------ */
/* Radial tables of one species: row-major nknots x 7 (radius, charge,
 * hartree, pot_P, pot_S, wfn_P, wfn_S) as V_ion/splineData.py:5-37; knots
 * pruned by V_ion/preProcess.py:4-26, natural cubic splines by
 * Splines/fspline.py:5-45.  zvalue/rcut: the Zvalue and R element columns. */
int psc_set_species(psc_ctx* ctx, int species_id, int nknots, const double* table, double zvalue, double rcut);
/* The host spline construction alone (pruning + coefficients), for checks. */
int psc_spline_coeffs(int nknots, const double* x, const double* y, int* nkeep, double* xk, double* z,
                      double* c, double* d);
/* SAD density, local pseudopotential and SAD Hartree potential:
 * V_ion/pseudoDiag.py:44-421 (backend.pseudo_diag, rsdft_solver.py:87).
 * species/xyz (host): natoms entries in species-major order, bohr.
 * h3 = h**3, fourpi = 4*pi, z_sum = sum of valence charges.
 * info[2] (host) = electron count before / after normalisation. */
int psc_sad_setup(psc_ctx* ctx, int natoms, const int* species, const double* xyz, double radius, double h3,
                  double fourpi, double z_sum, double* rho0, double* hpot0, double* ppot, double* info,
                  void* stream);
/* The density-file start (density_method = ml):
 * V_ion/pseudoDiag_ML4Den_poisson.py:392-530.  raw: the file's density
 * (1/A^3) flattened x-fastest on the device; rho1 = max(0, (raw a03) h3)
 * renormalised to z_sum (NumPy pairwise sums), hrhs = fourpi_h3 (rho1 - rho0).
 * info (host, 3, may be NULL): electron count after the unit conversion,
 * number of negative values set to 0, electron count after normalisation.
 * The ML-grid variants of the setup (pseudoDiag_MLgrid.py,
 * pseudoNL_original_MLgrid.py, pseudoNL_original_ML4Den.py) are
 * psc_sad_setup / psc_projector_setup with radius = 0: grid point i lies at
 * i h instead of i h - radius. */
int psc_ml_density(psc_ctx* ctx, const double* raw, double a03, double h3, double z_sum, const double* rho0,
                   double fourpi_h3, double* rho1, double* hrhs, double* info, void* stream);
/* Kleinman-Bylander projector tables (factored V_nl):
 * V_ion/pseudoNL_original.py:9-208 (backend.pseudo_nl, rsdft_solver.py:116). */
int psc_projector_setup(psc_ctx* ctx, int natoms, const int* species, const double* xyz, double radius,
                        void* stream);
/* Host copies of the projector tables (atom_off[atoms+1], idx[points],
 * u[3*points], w[atoms]); any pointer may be NULL. */
int psc_projector_export(psc_ctx* ctx, int* atom_off, int* idx, double* u, double* w);
/* np.sum order (pairwise) of a device vector, result on the device. */
int psc_numpy_sum(psc_ctx* ctx, const double* x, long n, double* out_dev, void* stream);

/* ---- Hamiltonian ------------------------------------------------------ */
/* Diagonal potential (Hartree, device, n): B = 0.5A + V_nl + diag(pot) at
 * rsdft_solver.py:285 without assembling B. */
int psc_set_potential(psc_ctx* ctx, const double* pot, void* stream);
/* Y = V_nl X alone: the factored form of the matrix pseudoNL returns
 * (V_ion/pseudoNL_original.py:187-206). */
int psc_apply_nonlocal(psc_ctx* ctx, int dtype, const void* X, long ldx, void* Y, long ldy, int k, void* stream);
/* Y = H X for k columns (the SpMM `H @ X` in the Eigensolvers package). */
int psc_apply_h(psc_ctx* ctx, int dtype, const void* X, long ldx, void* Y, long ldy, int k, void* stream);
/* Y = alpha H X + beta X + gamma P (P may be NULL or alias Y). */
int psc_apply_h_axpby(psc_ctx* ctx, int dtype, const void* X, long ldx, const void* P, long ldp, void* Y, long ldy,
                      int k, double alpha, double beta, double gamma, void* stream);
/* Stencil implementation: 0 = TMA-fed pipeline where the bulk-copy alignment
 * rules hold (default; 2-point FP64 runs, 4-point FP32 runs with the
 * arithmetic on packed pairs of points), 1 = register-queue kernel
 * everywhere, 2 = the TMA pipeline with 2-point FP32 runs when nx is even but
 * not a multiple of 4, 3 / 4 = as 2 / 0 with scalar FP32 arithmetic. */
int psc_set_stencil_impl(psc_ctx* ctx, int impl);
/* FP32 stencil weights.  Rounded to FP32 they break the sum rule
 * c0 + 6 sum c_d = 0 by a constant of order 1e-7 Ha that every eigenvalue
 * would carry.  2 (default) = the correction added to the FP32 potential
 * (pot32 = fl(pot + correction); a call with another potential, or none,
 * takes the term inside the TMA kernel); 1 = the correction as one more term
 * in the TMA kernel; 0 = plain FP32 weights.  Recasts the FP32 potential. */
int psc_set_stencil_weights(psc_ctx* ctx, int mode);
/* Sphere-masked Hamiltonian (no counterpart in the reference, which solves
 * on the whole cube): with radius > 0 (bohr) every H X returns zero at the
 * points farther than radius from the cube's centre, the projector tables
 * lose their points there, and the TMA stencil reads nothing for the planes
 * of a slab that hold no point inside (it only writes their zeros).  On
 * blocks that vanish outside the sphere this is P H P.  radius <= 0 restores
 * the cube.  Synchronises the stream. */
int psc_set_sphere_mask(psc_ctx* ctx, double radius, void* stream);
/* Zero the points outside the sphere mask in k columns (no-op without one). */
int psc_mask_block(psc_ctx* ctx, int dtype, void* X, long ld, int k, void* stream);
/* Y = A X with A = -Lap_h (Laplacian/fd3d.py:34-106 scaled by 1/h^2). */
int psc_laplacian_apply(psc_ctx* ctx, const double* x, double* y, int k, long ld, void* stream);

/* ---- eigensolver pieces ------------------------------------------------ */
/* Chebyshev filter of degree deg, bounds_dev = [lam1, low, high] on the
 * device.  mode 0: scaled filter Eigensolvers/ch_filter.py:4-81; mode 1:
 * cheb_filter_slim Eigensolvers/first_filt.py:78-103.  X holds the input and
 * is overwritten; *which = 0 if the result is in X, 1 if in Y. */
int psc_cheb_filter(psc_ctx* ctx, int dtype, int mode, int deg, const double* bounds_dev, void* X, void* Y,
                    long ld, int k, int* which, void* stream);
/* Six-step Lanczos bound.  mode 0: Eigensolvers/lancz_uppbnd.py:4-75,
 * out = [uppbnd, ritz_0..ritz_5]; mode 1: Eigensolvers/lanczosForChefsi1.py:5-99,
 * out = [bound].  The start vector is drawn from `seed`. */
int psc_lanczos_bound(psc_ctx* ctx, int mode, unsigned long long seed, double* out_dev, void* stream);
/* The same from the caller's start vector v_start (device, n doubles): the
 * vector lancz_uppbnd.py:22 draws (mode 0) or the one chefsi1.py:29 passes to
 * lanczosForChefsi1 (mode 1). */
int psc_lanczos_bound_v(psc_ctx* ctx, int mode, const double* v_start, double* out_dev, void* stream);
/* Lanczos with a kept basis (Eigensolvers/lanczosForChsubsp.py:33-119 and
 * lanczos.py:38-139, no reorthogonalisation): runs steps k0 .. k1-1 of
 * w = H v_j - beta_{j-1} v_{j-1}, alpha_j = v_j.w, w -= alpha_j v_j,
 * beta_j = |w|, v_{j+1} = w / beta_j.  VV (n x >= k1+1, column-major, ld
 * ldv) holds v_j in column j; ab[2j] = alpha_j, ab[2j+1] = beta_j (device).
 * With k0 = 0 the start vector is v_start / |v_start|, or a standard normal
 * vector drawn from `seed` when v_start is NULL (np.random.randn at
 * chsubsp.py:34 and rsdft_solver.py:63-68).  Calls with k0 > 0 continue a
 * run, so a caller can test convergence between them. */
int psc_lanczos_run(psc_ctx* ctx, const double* v_start, unsigned long long seed, int k0, int k1, double* VV,
                    long ldv, double* ab, void* stream);
/* Eigenpairs of the k x k symmetric tridiagonal with diagonal ab[2i] and
 * off-diagonal ab[2i+1] (k <= 4096): all eigenvalues ascending into evals,
 * eigenvectors of the nvec lowest into Z (k x nvec, ld ldz >= k) when
 * nvec > 0 (replaces scipy.linalg.eigh(Tmat[:k, :k]) at
 * lanczosForChsubsp.py:101-128 and lanczos.py:129-146). */
int psc_tridiag_eig(psc_ctx* ctx, const double* ab, int k, int nvec, double* evals, double* Z, long ldz,
                    void* stream);
/* Orthonormal basis of the numerically independent columns of W (n x k):
 * a column whose part orthogonal to the kept columns before it has squared
 * norm <= tol |w_j|^2 is dropped, the rest are orthonormalised by
 * CholeskyQR2.  *rank = kept columns, stored as the first *rank columns of W
 * (*which = 0) or T (*which = 1).  Replaces the Householder QR of
 * W = VV X at lanczosForChsubsp.py:167 and lanczos.py:195, whose input has
 * near-copies of the same Ritz vector. */
int psc_orthonormalize_rank(psc_ctx* ctx, int dtype, void* W, void* T, long ld, int k, double tol, int* rank,
                            int* which, void* stream);
/* Filter interval from device values: mode 0 chefsi1.py:29-38
 * ([min ritz, max ritz, upper]); mode 1 first_filt.py:28-29; mode 2 first_filt.py:62. */
int psc_filter_bounds(psc_ctx* ctx, int mode, const double* ritz_dev, int k, const double* upper_dev,
                      double* bounds_dev, void* stream);
/* Orthonormalise k columns by CholeskyQR applied `passes` times (replaces
 * scipy.linalg.qr at Eigensolvers/chefsi1.py:43 and first_filt.py:43). */
int psc_orthonormalize(psc_ctx* ctx, int dtype, void* W, void* T, long ld, int k, int passes, int* which,
                       void* stream);
/* Rayleigh-Ritz (chefsi1.py:46-67, first_filt.py:44-63): V = H W,
 * G = W^T H W (upper triangle mirrored), ascending eigenpairs, result W Q
 * written to V, Ritz values to ritz_dev. */
int psc_rayleigh_ritz(psc_ctx* ctx, int dtype, const void* W, void* V, long ld, int k, double* ritz_dev,
                      void* stream);
/* Rayleigh-Ritz of a filtered, not necessarily orthonormal block W in one
 * pass: V = H W, S = W^T W = R^T R, K = W^T V, eigenpairs of R^{-T} K R^{-1},
 * result W R^{-1} Y written to V (same Ritz pairs as QR followed by
 * Rayleigh-Ritz, chefsi1.py:43-67 / first_filt.py:43-63). */
int psc_subspace_rr(psc_ctx* ctx, int dtype, const void* W, void* V, long ld, int k, double* ritz_dev, void* stream);
/* Building blocks: G = A^T B (mode 0 plain, 1 upper mirrored, 2 symmetrised),
 * Out = W Q, symmetric eigensolver of (A + A^T)/2 (ascending, FP64,
 * Householder tridiagonalisation + bisection + inverse iteration, k <= 1024;
 * replaces scipy.linalg.eigh at first_filt.py:59 and chefsi1.py:64). */
int psc_gram(psc_ctx* ctx, int dtype, const void* A, long lda, const void* B, long ldb, int k, int mode,
             double* out_dev, void* stream);
int psc_gemm_nn(psc_ctx* ctx, int dtype, const void* W, long ldw, int k, const double* Q, int kout, void* out,
                long ldo, void* stream);
int psc_syev(psc_ctx* ctx, double* A, int k, double* evals, double* evecs, void* stream);
/* Fermi level and occupations by bisection: Eigensolvers/occupations.py:5-56
 * with Eigensolvers/FermiDirac.py:3-31 (backend.occupations, rsdft_solver.py:319). */
int psc_occupations(psc_ctx* ctx, const double* lam_dev, int n, double temp, double nelec, double tol,
                    double* ef_dev, double* occ_dev, void* stream);
/* rho = sum_i W_i^2 (2 f_i) / h^3 and hrhs = fourpi_h3 (h^3 rho - rho0)
 * (rsdft_solver.py:324-328); hrhs may be NULL.  For FP32 blocks each
 * orbital's weight is divided by its exact (FP64-summed) squared norm, so
 * that the electron count does not inherit the block's column-scale
 * rounding. */
int psc_density(psc_ctx* ctx, int dtype, const void* W, long ld, int nev, const double* occ_dev,
                const double* rho0, double fourpi_h3, double h3, double* rho, double* hrhs, void* stream);

/* ---- Hartree, XC, update, mixing ---------------------------------------- */
/* CG on A x = rhs, warm start in x (Eigensolvers/pcg.py:7-85, backend.pcg at
 * rsdft_solver.py:345). *its_out = iterations. */
int psc_pcg_poisson(psc_ctx* ctx, const double* rhs, double* x, int maxit, double tol, int* its_out, void* stream);
/* Preconditioned Hartree solve (cg_prec = 1): the preconditioned branch of
 * Eigensolvers/pcg.py:7-85 (stop when z.r <= tol^2 z0.r0), warm start in x,
 * with M = the inverse of the FD stencil continued by odd reflection across
 * the box faces, applied exactly by 3-D sine transforms.  It replaces the
 * ILU preconditioner of rsdft_solver.py:52-60,339, which the reference's CPU
 * path cannot apply (pcg.py:43 is handed the string "precLU") and its GPU
 * path ignores (pcg_gpu.py:38-41).  Grid dimensions up to 128.  The host
 * reads z.r once per iteration (these solves take a few iterations). */
int psc_pcg_poisson_prec(psc_ctx* ctx, const double* rhs, double* x, int maxit, double tol, int* its_out,
                         void* stream);
/* z = M r with the preconditioner above (r and z distinct device vectors). */
int psc_poisson_precond(psc_ctx* ctx, const double* r, double* z, void* stream);
/* CG execution mode: 2 (default) one persistent cooperative launch keeping
 * x, r, p, Ap in shared memory when they fit (else as 1); 1 the two CG
 * kernels replayed from a captured CUDA graph; 0 the two kernels launched from
 * the host.  All modes compute the same iterates. */
int psc_set_use_graphs(psc_ctx* ctx, int mode);
/* LDA (Ceperley-Alder / Perdew-Zunger), V_xc/exc_nspn.py:8-103.
 * out_dev = [exc, max rho, min rho]; max and min propagate NaN as numpy's
 * max and min do (rsdft_solver.py logs them). */
int psc_lda_xc(psc_ctx* ctx, const double* rho, double* vxc, double h3, double* out_dev, void* stream);
/* LDA exchange-correlation like psc_lda_xc, for callers that cannot allocate
 * device memory (inside a CUDA stream capture, or under a host that owns all
 * device memory through its own pool).  No counterpart in the reference: it
 * exists for those callers.  Needs no context and allocates nothing: its
 * per-CTA partials live in a fixed 96 KiB device array of the library.  rho,
 * vxc: n device doubles, 1 <= n <= 33554432 (larger n is rejected with
 * status 2); out_dev = [exc, max rho, min rho] (max and min propagate NaN,
 * as in psc_lda_xc).  The first call on a device looks up that array's
 * address and must come before any stream capture (a first call made during
 * a capture is refused with status 2); the address is kept for the process,
 * so do not call this entry point after cudaDeviceReset.  Concurrent calls
 * share the array and race, so serialise them. */
int psc_lda_xc_noalloc(const double* rho, double* vxc, long n, double h3, double* out_dev, void* stream);
/* pot_new = ppot + 0.5 vxc + hpot + hpot0, f = pot_new - pot (may be NULL),
 * out_dev = [|f|^2, |pot_new|^2, sum rho(hpot+hpot0), sum rho vxc]
 * (rsdft_solver.py:351-352 and :141-146). */
int psc_scf_update(psc_ctx* ctx, const double* ppot, const double* vxc, const double* hpot, const double* hpot0,
                   const double* rho, const double* pot, double* pot_new, double* f, double* out_dev, void* stream);
/* Multisecant Type-I mixer, group size 1: Mixer/mixer.py:169-217 and
 * Mixer/msecant1.py:40-175.  reset clears the history (capacity columns). */
int psc_mixer_reset(psc_ctx* ctx, int capacity);
int psc_mixer_step(psc_ctx* ctx, const double* x1, const double* f1, double mix, double restart_factor,
                   double* x_new, int* m_used, void* stream);
int psc_mixer_history(psc_ctx* ctx, int* m_out);
/* Type-II multisecant mixer (Mixer/msecant2.py:24-93; Anderson mixing with
 * group size 0): its control flow runs on the host, these are its operations
 * on the FP64 n-vectors of the history (n = the context's grid size, columns
 * lda apart, lda >= n):
 *   psc_mix2_diff:  df = f1 - df, dx = (x1 - dx) + mix df (msecant2.py:58-60)
 *   psc_mix2_store: dx = x1, df = f1
 *   psc_block_dots: out_dev[i] = A_i . x for the r columns of A
 *   psc_block_combine: y = base + mix f - sum_i A_i c_i (f may be NULL, y may
 *     be base)
 *   psc_block_absrow_max: out_dev[0] = max over rows of sum_i |A_i| (the
 *     infinity norm Mixer/qinv.py:27 scales its rank tolerance by).
 * The Gram matrix of a group and the product DF C use psc_gram and
 * psc_gemm_nn. */
int psc_mix2_diff(psc_ctx* ctx, const double* x1, const double* f1, double* dx, double* df, double mix,
                  void* stream);
int psc_mix2_store(psc_ctx* ctx, const double* x1, const double* f1, double* dx, double* df, void* stream);
int psc_block_dots(psc_ctx* ctx, const double* A, long lda, int r, const double* x, double* out_dev, void* stream);
int psc_block_combine(psc_ctx* ctx, double* y, const double* base, const double* f, double mix, const double* A,
                      long lda, int r, const double* c_dev, void* stream);
int psc_block_absrow_max(psc_ctx* ctx, const double* A, long lda, int r, double* out_dev, void* stream);

/* ---- utilities ---------------------------------------------------------- */
/* Counter-based random block: dist 0 uniform [0,1) (np.random.rand in
 * first_filt.py:37 and lancz_uppbnd.py:21), dist 1 standard normal
 * (np.random.randn in chefsi1.py:29). */
int psc_random(psc_ctx* ctx, int dtype, int dist, unsigned long long seed, void* out, long ld, long rows, int cols,
               void* stream);
int psc_cast(psc_ctx* ctx, int to_dtype, const void* src, void* dst, long n, void* stream);
/* out = a x + b y (y may be NULL), n doubles. */
int psc_axpby(psc_ctx* ctx, const double* x, const double* y, double a, double b, double* out, long n, void* stream);
/* Deterministic dot product, result on the device. */
int psc_dot(psc_ctx* ctx, const double* a, const double* b, long n, double* out_dev, void* stream);

/* Gram pairs of FP32 blocks (mixed precision) on tcgen05 tensor cores with
 * split-precision TF32 and FP32 accumulation (1, default) or on the FP64
 * tensor cores (DMMA) with exact products and FP64 accumulation (0, the path
 * of FP64 blocks).  No counterpart in the reference (its GPU path is cuBLAS
 * FP32). */
int psc_set_gram_impl(psc_ctx* ctx, int tensor_cores);
/* Rows per chunk of the tensor-core Gram pair (0 = automatic: four waves of
 * CTAs).  Each chunk accumulates in FP32 tensor memory, which rounds toward
 * zero; shorter chunks shrink that bias on the off-diagonal entries at the
 * cost of more partial tiles (at most 2 GiB). */
int psc_set_gram_chunk(psc_ctx* ctx, long rows);
/* Block products W T of FP32 blocks (the W Q of Rayleighritz.py:4-30 and
 * chefsi1.py:64-67, here W R^{-1} Y) on tcgen05 tensor cores with
 * split-precision TF32 and FP32 accumulation (1, default) or on the FP64
 * tensor cores (DMMA, FP64 products and sums, one rounding; 0).  No
 * counterpart in the reference (its GPU path is cuBLAS FP32). */
int psc_set_gemm_impl(psc_ctx* ctx, int tensor_cores);
/* S = W^T W and K = W^T V for n x k blocks (leading dimension ld), k x k
 * column-major FP64 results on the device (the Gram and projected-Hamiltonian
 * products of Rayleighritz.py:4-30). */
int psc_gram_pair(psc_ctx* ctx, int dtype, const void* W, const void* V, long ld, int k, double* S, double* K,
                  void* stream);

/* ---- learned initial density (3-D conv encoder-decoder) ------------------
 * No counterpart in the reference: it only consumes a predicted density
 * (V_ion/pseudoDiag_ML4Den_poisson.py:12-586, dispatched at
 * rsdft_solver.py:95-108).  Activations are channels-last BF16 [voxel][C]
 * (x fastest), C a multiple of 8; weights BF16 [tap][Cin][Cout] with
 * tap = dx + 3 (dy + 3 dz); biases and all gradients FP32; accumulation FP32.
 * geom[15] = {nxi, nyi, nzi, nxa, nya, nza, up, Ca, Cs, nxo, nyo, nzo,
 * stride, ksize, Cout}: the input is Ca channels of A (nearest-upsampled x2
 * when up = 1, A's grid is then the input grid halved, rounded up) followed by
 * Cs channels of the skip tensor S on the input grid; stride 1 or 2 (output
 * grid ceil(n / stride)), ksize 3 (padding 1) or 1. */
int psc_conv3d_fwd(psc_ctx* ctx, const int* geom, const void* A, const void* S, const void* W, const float* bias,
                   int act, void* out, float* out32, void* stream);
/* Forward implementation: 2 the tcgen05 implicit GEMM (BF16 operands, FP32
 * accumulation in tensor memory; activations 16-byte aligned), 0 the
 * CUDA-core kernel, 1 (default) by layer: tcgen05 from 32 output channels.
 * The backward always runs on the CUDA cores. */
int psc_set_conv_impl(psc_ctx* ctx, int impl);
/* act: 0 identity, 1 ReLU, 2 leaky ReLU (slope 1/16 below zero).
 * Backward of one convolution.  gout: dL/d(out) FP32 [nvo][Cout]; out: the
 * forward's BF16 output (needed when act != 0);
 * gm: FP32 scratch [nvo][Cout] (may alias gout); dvin: FP32 scratch
 * [nvi][Ca+Cs] or NULL to skip the input gradient; dA / dS: FP32 gradients of
 * A and S, overwritten (acc = 0) or accumulated (acc = 1), NULL to skip; dW,
 * dB: FP32 weight and bias gradients (overwritten); work: FP32 scratch of
 * work_floats (>= chunks x 27 Cin Cout). */
int psc_conv3d_bwd(psc_ctx* ctx, const int* geom, const void* A, const void* S, const void* W, const float* gout,
                   const void* out, int act, float* gm, float* dvin, float* dA, int acc_a, float* dS, int acc_s,
                   float* dW, float* dB, float* work, long work_floats, void* stream);
/* Mean squared error on channel 0 of y [n][C] against target [n]; grad [n][C]
 * = d loss / d y; loss_dev = one double on the device. */
int psc_mse_loss(psc_ctx* ctx, const float* y, int C, const float* target, long n, float* grad, double* loss_dev,
                 void* stream);
/* Adam step on FP32 master weights w (n), refreshing the BF16 copy wb (may be
 * NULL); step counts from 1. */
int psc_adam_step(psc_ctx* ctx, float* w, void* wb, const float* grad, float* m, float* v, long n, float lr,
                  float b1, float b2, float eps, int step, void* stream);
int psc_f32_to_bf16(psc_ctx* ctx, const float* x, void* y, long n, void* stream);
/* Network input on the context's grid: BF16 [n][8], ch0 = a0 x0, ch1 = a1 x1, rest 0. */
int psc_pack_input(psc_ctx* ctx, const double* x0, const double* x1, double a0, double a1, void* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PSC_H */
