/* Matrix-free finite-difference apply for the CPU oracle (TEST INFRASTRUCTURE).
 *
 * This file checks the product and is never part of it.  It is compiled into
 * oracle/liboracle_fd.so and loaded only by oracle/oracle.py, which the tests,
 * the smoke check and the CPU legs of bench.py import.
 *
 * It computes, for a block of k grid vectors on the nx x ny x nz cube with
 * flat index p = i + nx (j + ny l) and zero values outside the cube,
 *
 *     Y[:, c] = scale * (A X[:, c]) + pot .* X[:, c]
 *
 * where A is the star stencil of Laplacian/fd3d.py:34-106 (centre weight
 * w[0], weights w[1..R] of the offsets +-1..+-R along each axis, 3 w[0]
 * summed in the centre; the caller passes the per-axis weights and the
 * centre weight already tripled).  scale = 1/h^2 gives the matrix of
 * rsdft_solver.py:186; scale = 0.5/h^2 with pot the local potential gives the
 * local part of H = 0.5 A + diag(pot) of rsdft_solver.py:263,285.  The same
 * numbers as the reference's CSR product up to the order of the sums.
 *
 * Two layouts: column-major blocks (point stride 1, column stride ld) and
 * point-major blocks (point stride k, column stride 1, NumPy's C-order n x k
 * arrays).  Threads split the z planes (and the columns of column-major
 * blocks) with OpenMP.
 */
#include <stddef.h>

static void col_major(long nx, long ny, long nz, int R, const double *w, double scale, const double *pot,
                      const double *X, long ldx, double *Y, long ldy, long k)
{
    const long pl = nx * ny;
#pragma omp parallel for collapse(2) schedule(static)
    for (long c = 0; c < k; ++c) {
        for (long z = 0; z < nz; ++z) {
            const double *x = X + c * ldx;
            double *y = Y + c * ldy;
            for (long yy = 0; yy < ny; ++yy) {
                const long row = z * pl + yy * nx;
                for (long i = 0; i < nx; ++i) {
                    const long p = row + i;
                    double acc = w[0] * x[p];
                    for (int d = 1; d <= R; ++d) {
                        double s = 0.0;
                        if (i - d >= 0) s += x[p - d];
                        if (i + d < nx) s += x[p + d];
                        if (yy - d >= 0) s += x[p - d * nx];
                        if (yy + d < ny) s += x[p + d * nx];
                        if (z - d >= 0) s += x[p - d * pl];
                        if (z + d < nz) s += x[p + d * pl];
                        acc += w[d] * s;
                    }
                    double v = scale * acc;
                    if (pot) v += pot[p] * x[p];
                    y[p] = v;
                }
            }
        }
    }
}

static void point_major(long nx, long ny, long nz, int R, const double *w, double scale, const double *pot,
                        const double *X, double *Y, long k)
{
    const long pl = nx * ny;
#pragma omp parallel for schedule(static)
    for (long z = 0; z < nz; ++z) {
        for (long yy = 0; yy < ny; ++yy) {
            for (long i = 0; i < nx; ++i) {
                const long p = z * pl + yy * nx + i;
                double *y = Y + p * k;
                const double *xc = X + p * k;
                for (long c = 0; c < k; ++c) y[c] = w[0] * xc[c];
                for (int d = 1; d <= R; ++d) {
                    const double wd = w[d];
                    long nb[6];
                    int m = 0;
                    if (i - d >= 0) nb[m++] = p - d;
                    if (i + d < nx) nb[m++] = p + d;
                    if (yy - d >= 0) nb[m++] = p - d * nx;
                    if (yy + d < ny) nb[m++] = p + d * nx;
                    if (z - d >= 0) nb[m++] = p - d * pl;
                    if (z + d < nz) nb[m++] = p + d * pl;
                    for (int q = 0; q < m; ++q) {
                        const double *xn = X + nb[q] * k;
                        for (long c = 0; c < k; ++c) y[c] += wd * xn[c];
                    }
                }
                const double pp = pot ? pot[p] : 0.0;
                for (long c = 0; c < k; ++c) y[c] = scale * y[c] + pp * xc[c];
            }
        }
    }
}

/* layout 0: column-major (ldx, ldy leading dimensions); 1: point-major (k
 * values per point, contiguous).  pot may be NULL.  Returns 0, or 2 on a bad
 * argument. */
int oracle_fd_apply(long nx, long ny, long nz, int R, const double *w, double scale, const double *pot,
                    const double *X, long ldx, double *Y, long ldy, long k, int layout)
{
    if (nx <= 0 || ny <= 0 || nz <= 0 || R < 1 || R > 8 || k < 0 || !w || !X || !Y) return 2;
    if (layout == 0) {
        if (ldx < nx * ny * nz || ldy < nx * ny * nz) return 2;
        col_major(nx, ny, nz, R, w, scale, pot, X, ldx, Y, ldy, k);
        return 0;
    }
    if (layout == 1) {
        point_major(nx, ny, nz, R, w, scale, pot, X, Y, k);
        return 0;
    }
    return 2;
}
