"""CPU oracle for the real-space Kohn-Sham SCF hot path (TEST INFRASTRUCTURE).

This module checks the product and is never part of it.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` may import
it.  The product path (``parsec_python_b200``) runs on the GPU through
``libpsc.so`` and never calls into this file.

It restates, in NumPy/SciPy, the algorithm of PARSEC.py's CPU path
(zeyizhang-berkeley/parsec_python, ``src/``).  Each function cites the
reference file:line it follows.  Where the reference has a quirk that changes
numbers (the aliased first search direction in ``pcg``, the beta rescale in
``lancz_uppbnd``, the zero-padded tridiagonal in the same routine) the quirk is
kept, because parity means "the same numbers as the reference".

The restatement deliberately builds the same CSR Hamiltonian as the reference
(``0.5*A + V_nl + diag(pot)`` with ``A = (1/h^2) * fd3d``) and makes the same
``numpy.random`` calls in the same order, so that with the same global seed the
oracle reproduces the reference's SCF trajectory to rounding.  It is pinned
against fixtures generated by running the reference itself
(``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import scipy.linalg
import scipy.sparse as sp

A0_ANG = 0.529177210903     # rsdft_models.py:14
RY_EV = 13.605698066        # rsdft_models.py:15

_DATA = Path(__file__).resolve().parents[1] / "parsec_python_b200" / "data"


# ----------------------------------------------------------------------------
# data tables
# ----------------------------------------------------------------------------
def load_elements(path: Path | None = None) -> dict:
    """Element defaults; columns as in rsdft_input.py:23-31."""
    path = Path(path or _DATA / "elements.csv")
    out = {}
    for order, line in enumerate(path.read_text().splitlines()):
        if not line.strip():
            continue
        f = line.split(",")
        out[f[0]] = {"order": order, "AtomicNumber": int(f[1]), "Z": int(f[2]),
                     "Zvalue": float(f[3]), "h": float(f[4]), "r": float(f[5]),
                     "R": float(f[6])}
    return out


def load_tables(path: Path | None = None) -> dict:
    """Radial tables (radius, charge, hartree, pot_P, pot_S, wfn_P, wfn_S);
    V_ion/splineData.py:5-37."""
    with np.load(path or _DATA / "pseudo_tables.npz") as z:
        return {k: z[k] for k in z.files}


# ----------------------------------------------------------------------------
# splines (Splines/fspline.py, Splines/fsplevalIO.py, Splines/trid.py,
# V_ion/preProcess.py)
# ----------------------------------------------------------------------------
def prune_knots(v: np.ndarray) -> np.ndarray:
    """Keep knot 0, every knot whose value moved by more than 1e-5 from the
    previous raw knot, and the last knot.  V_ion/preProcess.py:4-26."""
    v = np.asarray(v)
    keep = np.abs(v[1:-1] - v[:-2]) > 10e-6
    return np.concatenate([[0], np.nonzero(keep)[0] + 1, [len(v) - 1]])


def spline_coeffs(xi: np.ndarray, yi: np.ndarray):
    """Natural cubic spline in the (z, c, d) form of Splines/fspline.py:5-45,
    tridiagonal solve by Splines/trid.py:3-32 (sequential Thomas sweep)."""
    xi = np.asarray(xi, dtype=np.float64).ravel()
    yi = np.asarray(yi, dtype=np.float64).ravel()
    n = len(xi) - 1
    h = xi[1:] - xi[:-1]
    r = (yi[1:] - yi[:-1]) / h
    r = (r[1:n] - r[0:n - 1]).tolist()
    a = h[0:n - 1].tolist()
    c = h[1:n].tolist()
    d = (2 * (h[0:n - 1] + h[1:n])).tolist()
    m = len(d)
    for k in range(1, m):
        piv = a[k] / d[k - 1]
        d[k] = d[k] - piv * c[k - 1]
        r[k] = r[k] - piv * r[k - 1]
    r[m - 1] = r[m - 1] / d[m - 1]
    for j in range(m - 2, -1, -1):
        r[j] = (r[j] - c[j] * r[j + 1]) / d[j]
    z = np.concatenate([[0.0], np.array(r), [0.0]])
    cc = (yi[0:n] / h) - (z[0:n] * h)
    dd = (yi[1:] / h) - (z[1:] * h)
    return z, cc, dd


class Spline:
    """Knots + coefficients with the evaluation rule of Splines/fsplevalIO.py:2-65:
    clamp x to [xi[0], xi[-1]], pick the interval [xi[j], xi[j+1]] containing x
    (binary search convention: largest j with xi[j] <= x, at most n-2), then
    y = t1*(z_j*t1*t1/h_j + c_j) + t2*(z_{j+1}*t2*t2/h_j + d_j).

    The reference warm-starts the search from the previous point's interval;
    that can only pick a different (adjacent) interval when x equals a knot
    exactly, where both intervals give the same value up to rounding."""

    def __init__(self, xi, yi):
        self.xi = np.asarray(xi, dtype=np.float64)
        self.z, self.c, self.d = spline_coeffs(self.xi, yi)

    def __call__(self, x):
        xi = self.xi
        x = np.clip(np.asarray(x, dtype=np.float64), xi[0], xi[-1])
        j = np.searchsorted(xi, x, side="right") - 1
        j = np.clip(j, 0, len(xi) - 2)
        t1 = xi[j + 1] - x
        t2 = x - xi[j]
        hj = xi[j + 1] - xi[j]
        return t1 * (self.z[j] * t1 * t1 / hj + self.c[j]) + t2 * (self.z[j + 1] * t2 * t2 / hj + self.d[j])


def pruned_spline(r, y) -> Spline:
    idx = prune_knots(y)
    return Spline(r[idx], y[idx])


# ----------------------------------------------------------------------------
# grid, Laplacian
# ----------------------------------------------------------------------------
def fd_stencil(order: int):
    """Centre weight and per-offset weights of -h^2 * d2/dx2 summed over the
    three axes; Laplacian/fd3d.py:49-94 (orders <=2, <=4, <=6, else 8)."""
    if order <= 2:
        return 6.0, (-1.0,)
    if order <= 4:
        return 15 / 2, (-4 / 3, 1 / 12)
    if order <= 6:
        return 49 / 6, (-3 / 2, 3 / 20, -1 / 90)
    return 205 / 24, (-8 / 5, 1 / 5, -8 / 315, 1 / 560)


def fd3d(nx: int, ny: int, nz: int, order: int) -> sp.csr_matrix:
    """Sparse -h^2*Laplacian with zero Dirichlet values outside the cube,
    flat index p = i + nx*(j + ny*k).  Same entries as Laplacian/fd3d.py:34-106
    (duplicate diagonals of tiny grids summed)."""
    c0, cs = fd_stencil(order)
    n = nx * ny * nz
    p = np.arange(n)
    i = p % nx
    j = (p // nx) % ny
    k = p // (nx * ny)
    rows, cols, vals = [p], [p], [np.full(n, c0)]
    for d, cd in enumerate(cs, start=1):
        for coord, ext, stride in ((i, nx, 1), (j, ny, nx), (k, nz, nx * ny)):
            ok = coord + d < ext
            a = p[ok]
            b = a + d * stride
            rows += [a, b]
            cols += [b, a]
            vals += [np.full(a.size, cd), np.full(a.size, cd)]
    m = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return m.tocsr()


def laplacian(domain: dict, order: int) -> sp.csr_matrix:
    """A = (1/h^2) * fd3d, rsdft_solver.py:186."""
    h = domain["h"]
    return ((1.0 / (h * h)) * fd3d(domain["nx"], domain["ny"], domain["nz"], order)).tocsr()


# ----------------------------------------------------------------------------
# ionic setup
# ----------------------------------------------------------------------------
def pseudo_diag(domain: dict, atoms: list, elements: dict, tables: dict):
    """Superposition of atomic densities (SAD), local pseudopotential and the
    SAD Hartree potential.  V_ion/pseudoDiag.py:44-421.

    Per atom, in species then atom order, and per grid point:
    ppot += S_potS(r), rho0 += max(0, S_charge(r) * h^3 / (4 pi)),
    hpot0 += S_hartree(r), with r^2 = (dz^2 + dy^2) + dx^2 (pseudoDiag.py:203-212);
    finally rho0 <- Z_sum * rho0 / sum(rho0) (pseudoDiag.py:293-297).
    Returns (rho0, hpot0, ppot, info)."""
    nx, ny, nz, h, rad = domain["nx"], domain["ny"], domain["nz"], domain["h"], domain["radius"]
    n = nx * ny * nz
    pot = np.zeros(n)
    rho0 = np.zeros(n)
    hpot0 = np.zeros(n)
    z_sum = 0.0
    for species in atoms:
        typ, xyz = species["typ"], np.asarray(species["coord"], dtype=np.float64)
        z_sum += elements[typ]["Z"] * xyz.shape[0]
        data = tables[typ]
        s_chg = pruned_spline(data[:, 0], data[:, 1])
        s_pot = pruned_spline(data[:, 0], data[:, 4])
        s_hrt = pruned_spline(data[:, 0], data[:, 2])
        for a in range(xyz.shape[0]):
            dz = (np.arange(nz) * h - rad - xyz[a, 2]) ** 2
            dy = (np.arange(ny) * h - rad - xyz[a, 1]) ** 2
            dx = (np.arange(nx) * h - rad - xyz[a, 0]) ** 2
            r = np.sqrt((dz[:, None, None] + dy[None, :, None]) + dx[None, None, :]).ravel()
            pot += s_pot(r)
            rho0 += np.maximum(0, s_chg(r) * (h ** 3) / (4 * np.pi))
            hpot0 += s_hrt(r)
    rho0_sum = np.sum(rho0)
    info = {"electron_count_initial": float(rho0_sum)}
    rho0 = z_sum * rho0 / rho0_sum
    info["electron_count_normalized"] = float(np.sum(rho0))
    info["electron_target"] = float(z_sum)
    return rho0, hpot0, pot, info


def projectors(domain: dict, atoms: list, elements: dict, tables: dict) -> list:
    """Kleinman-Bylander p-channel projectors in factored form.
    V_ion/pseudoNL_original.py:9-208.

    For each atom: window of grid points [i0-span, i0+span] (1-based, clipped)
    with i0 = round((x + rad)/h + 1), span = round(R/h) (Python half-even
    rounding), points with 0 < |r| < R (|r|^2 = (dx^2 + dy^2) + dz^2), and
    u_m = (r_m/|r|) * wfn_P(|r|) * (pot_P - pot_S)(|r|), m = x, y, z.
    V_nl = sum_atoms sum_m u_m u_m^T / xint with xint = Zvalue / h^3.
    Returns a list of dicts {idx (0-based flat), u (3, n_a), xint}."""
    nx, ny, nz, h, rad = domain["nx"], domain["ny"], domain["nz"], domain["h"], domain["radius"]
    out = []
    for species in atoms:
        typ, xyz = species["typ"], np.asarray(species["coord"], dtype=np.float64)
        data = tables[typ]
        xi = data[:, 0]
        pot_ps = data[:, 3] - data[:, 4]
        wfn_p = data[:, 5]
        s_wfn = pruned_spline(xi, wfn_p)
        s_pps = pruned_spline(xi, pot_ps)
        xint = elements[typ]["Zvalue"] / (h ** 3)
        r0 = elements[typ]["R"]
        for a in range(xyz.shape[0]):
            xxa, yya, zza = float(xyz[a, 0]), float(xyz[a, 1]), float(xyz[a, 2])
            i0 = int(round((xxa + rad) / h + 1))
            j0 = int(round((yya + rad) / h + 1))
            k0 = int(round((zza + rad) / h + 1))
            span = int(round(r0 / h))
            imin, imax = max(1, i0 - span), min(nx, i0 + span)
            jmin, jmax = max(1, j0 - span), min(ny, j0 + span)
            kmin, kmax = max(1, k0 - span), min(nz, k0 + span)
            if imin > imax or jmin > jmax or kmin > kmax:
                continue
            kk, jj, ii = np.meshgrid(np.arange(kmin, kmax + 1), np.arange(jmin, jmax + 1),
                                     np.arange(imin, imax + 1), indexing="ij")
            kk, jj, ii = kk.ravel(), jj.ravel(), ii.ravel()
            xxx = (ii - 1) * h - rad - xxa
            yyy = (jj - 1) * h - rad - yya
            zzz = (kk - 1) * h - rad - zza
            dd = np.sqrt(xxx ** 2 + yyy ** 2 + zzz ** 2)
            m = (dd > 0) & (dd < r0)
            if not np.any(m):
                continue
            xxx, yyy, zzz, dd = xxx[m], yyy[m], zzz[m], dd[m]
            idx = (ii[m] - 1) + nx * ((jj[m] - 1) + (kk[m] - 1) * ny)
            vspp = s_pps(dd)
            wavpp = s_wfn(dd)
            u = np.stack([xxx / dd * wavpp * vspp, yyy / dd * wavpp * vspp, zzz / dd * wavpp * vspp])
            out.append({"idx": idx.astype(np.int64), "u": u, "xint": float(xint), "typ": typ})
    return out


def ml_grid(domain: dict) -> dict:
    """The ML-grid setups (V_ion/pseudoDiag_MLgrid.py, pseudoNL_original_MLgrid.py,
    pseudoNL_original_ML4Den.py) are the SAD ones with grid point i at i h
    instead of i h - radius: the same arithmetic with the radius 0."""
    return dict(domain, radius=0.0)


def ml_density_start(domain: dict, atoms: list, elements: dict, tables: dict, density, order: int = 8,
                     cg_prec: int = 0):
    """The density-file start, V_ion/pseudoDiag_ML4Den_poisson.py:12-586:
    SAD on the ML grid; rho1 = ravel_F(density a0^3) h^3 (density in 1/A^3),
    negatives set to 0, renormalised to Z_sum; the Hartree potential of
    rho1 - rho0 by CG from zero (tol 1e-5, 200 iterations) added to the SAD
    one.  Returns (rho1, hpot1, ppot, info)."""
    rho0, hpot0, ppot, _ = pseudo_diag(ml_grid(domain), atoms, elements, tables)
    h = domain["h"]
    z_sum = 0.0
    for a in atoms:
        z_sum += elements[a["typ"]]["Z"] * np.asarray(a["coord"]).reshape(-1, 3).shape[0]
    rho1 = np.ravel(np.asarray(density, dtype=np.float64) * (A0_ANG ** 3), order="F") * (h ** 3)
    count0 = float(np.sum(rho1))
    rho1[rho1 < 0] = 0.0
    rho1 = z_sum * rho1 / np.sum(rho1)
    hrhs = (4 * np.pi / h ** 3) * (rho1 - rho0)
    A = laplacian(domain, order)
    if cg_prec:
        dh, _ = pcg_prec(A, hrhs, np.zeros(rho1.size), 200, 1e-5, spectral_preconditioner(domain, order))
    else:
        dh, _ = pcg(A, hrhs, np.zeros(rho1.size), 200, 1e-5)
    info = {"electron_count_initial": count0, "electron_count_normalized": float(np.sum(rho1)),
            "electron_target": float(z_sum)}
    return rho1, dh + hpot0, ppot, info


def nonlocal_csr(projs: list, n: int) -> sp.csr_matrix:
    """Assemble V_nl as the reference does (dense per-atom blocks
    outer(ux,ux)/xint + outer(uy,uy)/xint + outer(uz,uz)/xint summed over
    atoms), pseudoNL_original.py:187-206."""
    vnl = sp.csr_matrix((n, n))
    for pr in projs:
        ux, uy, uz = pr["u"]
        xint = pr["xint"]
        total = np.outer(ux, ux) / xint + np.outer(uy, uy) / xint + np.outer(uz, uz) / xint
        idx = pr["idx"]
        r = np.repeat(idx, idx.size)
        c = np.tile(idx, idx.size)
        vnl = vnl + sp.coo_matrix((total.ravel(), (r, c)), shape=(n, n)).tocsr()
    return vnl.tocsr()


def nonlocal_apply(projs: list, x: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
    """Factored V_nl @ x = sum_a sum_m u_m (u_m . x[idx]) / xint, added to
    `out` when given (pseudoNL_original.py:187-206 without forming the
    n x n matrix)."""
    y = np.zeros_like(x) if out is None else out
    for pr in projs:
        idx, u = pr["idx"], pr["u"]
        proj = u @ x[idx]                      # (3, k)
        y[idx] += (u.T @ proj) / pr["xint"]
    return y


_FD_LIB = None


def _fd_lib():
    """oracle/liboracle_fd.so (oracle/fd_apply.c), built on first use."""
    global _FD_LIB
    if _FD_LIB is None:
        import ctypes

        from oracle import build_oracle

        lib = ctypes.CDLL(str(build_oracle.build()))
        lib.oracle_fd_apply.restype = ctypes.c_int
        lib.oracle_fd_apply.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long,
                                        ctypes.c_void_p, ctypes.c_long, ctypes.c_long, ctypes.c_int]
        _FD_LIB = lib
    return _FD_LIB


def fd_apply(domain: dict, order: int, x: np.ndarray, scale: float, pot: np.ndarray | None = None) -> np.ndarray:
    """scale * (fd3d @ x) + pot * x, matrix-free (oracle/fd_apply.c), for a
    vector (n,) or a block (n, k) in C or Fortran order; the result has the
    layout of x.  The same stencil as fd3d (Laplacian/fd3d.py:34-106) with
    the sums in a different order."""
    import ctypes

    nx, ny, nz = domain["nx"], domain["ny"], domain["nz"]
    n = nx * ny * nz
    c0, cs = fd_stencil(order)
    w = np.ascontiguousarray([c0] + list(cs), dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    if x.shape[0] != n:
        raise ValueError(f"operand has {x.shape[0]} rows, the grid {n} points")
    if x.ndim == 1 or x.flags.f_contiguous:
        layout = 0
    elif x.flags.c_contiguous:
        layout = 1
    else:
        x = np.ascontiguousarray(x)
        layout = 1
    k = 1 if x.ndim == 1 else x.shape[1]
    y = np.empty_like(x)
    p = None if pot is None else np.ascontiguousarray(pot, dtype=np.float64)
    vp = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    st = _fd_lib().oracle_fd_apply(nx, ny, nz, len(cs), vp(w), float(scale), vp(p), vp(x), n, vp(y), n, k, layout)
    if st != 0:
        raise ValueError("oracle_fd_apply: invalid argument")
    return y


class StencilLaplacian:
    """A = (1/h^2) fd3d (rsdft_solver.py:186) as an operator: A @ x and
    A.dot(x) give the CSR product of laplacian() up to the order of sums."""

    def __init__(self, domain: dict, order: int):
        self.domain, self.order = domain, order
        n = domain["nx"] * domain["ny"] * domain["nz"]
        self.shape = (n, n)

    def dot(self, x):
        return fd_apply(self.domain, self.order, x, 1.0 / self.domain["h"] ** 2)

    __matmul__ = dot


class StencilHamiltonian:
    """B = 0.5 A + V_nl + diag(pot) (rsdft_solver.py:263,285) as an
    operator: the stencil and the local potential in one C pass, then the
    factored projectors.  The same numbers as the assembled CSR B up to the
    order of sums; used for the largest configurations, whose CSR products
    take minutes per block on the host."""

    def __init__(self, domain: dict, order: int, projs: list, pot: np.ndarray):
        self.domain, self.order, self.projs = domain, order, projs
        self.pot = np.ascontiguousarray(pot, dtype=np.float64)
        n = self.pot.size
        self.shape = (n, n)

    def dot(self, x):
        y = fd_apply(self.domain, self.order, x, 0.5 / self.domain["h"] ** 2, self.pot)
        return nonlocal_apply(self.projs, np.asarray(x, dtype=np.float64), out=y)

    __matmul__ = dot


def nuclear(atoms: list, elements: dict) -> float:
    """E_nuc = 2 * sum_{i<j} Z_i Z_j / R_ij (Ry), Laplacian/nuclear.py:26-91."""
    xs, zs = [], []
    for species in atoms:
        xyz = np.asarray(species["coord"], dtype=np.float64)
        for a in range(xyz.shape[0]):
            xs.append(xyz[a])
            zs.append(elements[species["typ"]]["Z"])
    e = 0
    for i in range(len(xs)):
        for j in range(i + 1, len(xs)):
            d2 = (xs[i][0] - xs[j][0]) ** 2 + (xs[i][1] - xs[j][1]) ** 2 + (xs[i][2] - xs[j][2]) ** 2
            e += zs[i] * zs[j] / np.sqrt(d2)
    return float(e * 2)


def nelectrons(atoms: list, elements: dict) -> int:
    """V_ion/nelectrons.py:1-23."""
    return sum(len(s["coord"]) * elements[s["typ"]]["Z"] for s in atoms)


# ----------------------------------------------------------------------------
# exchange-correlation
# ----------------------------------------------------------------------------
def exc_nspn(h: float, rho: np.ndarray):
    """Ceperley-Alder / Perdew-Zunger LDA, V_xc/exc_nspn.py:8-103.
    Returns (vxc [Ry], exc [Ry] = h^3 * sum(0.75 rho v_x + rho eps_c))."""
    g, b1, b2 = -0.2846, 1.0529, 0.3334
    c1, c2, c3, c4, c5 = 0.0622, 0.096, 0.004, 0.0232, 0.0192
    third = 1.0 / 3.0
    a0 = (4.0 / (9.0 * np.pi)) ** third
    twovpia0 = 2.0 / (np.pi * a0)
    p75vpi = 0.75 / np.pi
    rho = np.asarray(rho, dtype=np.float64)
    vxc = np.zeros_like(rho)
    pos = rho > 0
    rv = rho[pos]
    rs = (p75vpi / rv) ** third
    vx = -twovpia0 / rs
    ec = np.empty_like(rs)
    vc = np.empty_like(rs)
    hi = rs >= 1.0
    sq = np.sqrt(rs[hi])
    ec[hi] = g / (1.0 + b1 * sq + b2 * rs[hi])
    vc[hi] = (ec[hi] ** 2) * (1.0 + 3.5 * b1 * sq * third + 4.0 * b2 * rs[hi] * third) / g
    lo = ~hi
    al = np.log(rs[lo])
    ec[lo] = c1 * al - c2 + (c3 * al - c4) * rs[lo]
    vc[lo] = ec[lo] - (c1 + (c3 * al - c5) * rs[lo]) * third
    vxc[pos] = vx + vc
    exc = float(np.sum(0.75 * rv * vx + rv * ec)) * h ** 3
    return vxc, exc


# ----------------------------------------------------------------------------
# eigensolver pieces (Eigensolvers/)
# ----------------------------------------------------------------------------
def _gram_upper(vin: np.ndarray, w: np.ndarray) -> np.ndarray:
    """G[i,j] = Vin_i . W_j for i <= j, mirrored (first_filt.py:53-57,
    chefsi1.py:51-54)."""
    m = vin.T @ w
    return np.triu(m) + np.triu(m, 1).T


def lancz_uppbnd(n: int, A, k: int = 6):
    """Eigensolvers/lancz_uppbnd.py:4-75, including the beta *= 10 rescale that
    feeds the next step and the zero-padded (j+1)x(j+1) tridiagonal."""
    k = min(max(k, 6), 10)
    T = np.zeros((k, k))
    v = np.random.rand(n, 1)
    v = v / np.linalg.norm(v)
    tol = 2.5e-16
    upperb = np.zeros((3, k))
    f = A @ v
    alpha = np.vdot(v, f)
    f = f - alpha * v
    T[0, 0] = alpha
    beta = np.linalg.norm(f)
    upperb[:, 0] = alpha + beta
    ritzv = None
    X = None
    j = 1
    for j in range(2, k + 1):
        if beta > tol:
            v0 = v
            v = f / beta
            f = A @ v
            f = f - beta * v0
            alpha = np.vdot(v, f)
            f = f - alpha * v
            T[j - 1, j - 2] = beta
            T[j - 2, j - 1] = beta
            T[j - 1, j - 1] = alpha
        else:
            break
        beta = np.linalg.norm(f)
        ritzv, X = scipy.linalg.eigh(T[0:j + 1, 0:j + 1])
        if beta < 1e-2:
            beta = beta * 10
        upperb[0, j - 1] = ritzv[-1] + beta
        upperb[1, j - 1] = ritzv[-1] + abs(X[-1, -1]) * beta
        upperb[2, j - 1] = ritzv[-1] + max(abs(X[-1, :])) * beta
    uppbnd = (upperb[0, j - 1] + upperb[1, j - 1]) / 2
    uppbnd = (upperb[2, j - 1] + uppbnd) / 2
    return uppbnd, ritzv


def lanczos_bound(B, v) -> float:
    """Six-step Lanczos bound max|theta| + beta_6;
    Eigensolvers/lanczosForChefsi1.py:5-99 with nev = m = 6, tol = 0."""
    m = 6
    n = B.shape[0]
    v = v / np.linalg.norm(v)
    v1 = v
    v0 = np.zeros((n, 1))
    bet = 0
    T = np.zeros((m + 1, m + 1))
    for kk in range(1, m + 1):
        v = B @ v1 - bet * v0
        alp = np.vdot(v1, v)
        v = v - alp * v1
        bet = np.linalg.norm(v)
        v0 = v1
        v1 = v / bet
        T[kk - 1, kk - 1] = alp
        T[kk, kk - 1] = bet
        T[kk - 1, kk] = bet
    rr = np.sort(scipy.linalg.eigh(T[:m, :m], eigvals_only=True))
    return float(max(np.abs(rr)) + bet)


def cheb_filter_slim(H, x, polm, low, high):
    """Unscaled Chebyshev filter, Eigensolvers/first_filt.py:78-103."""
    e = (high - low) / 2
    center = (high + low) / 2
    y = H @ x
    y = (-y + center * x) / e
    for _ in range(2, polm + 1):
        ynew = H @ y
        ynew = (-ynew + center * y) * 2 / e - x
        x = y
        y = ynew
    return y


def ch_filter(A, x, deg, lam1, low, high):
    """Scaled Chebyshev filter, Eigensolvers/ch_filter.py:4-81."""
    e = (high - low) / 2
    c = (high + low) / 2
    sigma1 = e / (lam1 - c)
    sigma = sigma1
    y = (A @ x - c * x) * (sigma1 / e)
    two_over_s1 = 2.0 / sigma1
    inv_e = 1.0 / e
    for _ in range(2, deg + 1):
        sigma_new = 1.0 / (two_over_s1 - sigma)
        t1 = 2.0 * sigma_new * inv_e
        t2 = sigma * sigma_new
        ynew = (A @ y - c * y) * t1 - t2 * x
        x = y
        y = ynew
        sigma = sigma_new
    return y


def first_filt(nev: int, H, polm: int = 10):
    """First SCF step: random block + filter + RR rounds,
    Eigensolvers/first_filt.py:6-75."""
    energ_tol = 0.08
    if polm < 10 or polm > 15:
        polm = 10
    max_iter = max(min(int(60 / polm), 5), 3)
    n = H.shape[0]
    upperb, ritzv = lancz_uppbnd(n, H)
    lowerb = 0.8 * ritzv[0] + 0.2 * ritzv[-2]
    W = np.random.rand(n, nev)
    tr0 = 0.0
    for it in range(1, max_iter + 1):
        W = cheb_filter_slim(H, W, polm, lowerb, upperb)
        W, _ = scipy.linalg.qr(W, mode="economic", pivoting=False)
        Vin = H @ W
        G = _gram_upper(Vin, W)
        ritzv_raw, Q = scipy.linalg.eigh(G)
        order = np.argsort(ritzv_raw)
        ritzv = ritzv_raw[order]
        lowerb = ritzv[-1]
        W = W @ Q[:, order]
        if it == 1:
            tr0 = np.sum(ritzv[:nev])
        else:
            tr1 = np.sum(ritzv[:nev])
            if abs(tr1 - tr0) <= energ_tol * abs(tr0):
                break
            tr0 = tr1
    return W, ritzv


def chefsi1(Vin, ritzv, deg, nev, H):
    """One Chebyshev-filtered subspace step, Eigensolvers/chefsi1.py:10-69."""
    n, n2 = Vin.shape
    if nev >= n2:
        raise ValueError("Vin should have more than nev columns")
    upperb = lanczos_bound(H, np.random.randn(n, 1))
    lowerb = np.max(ritzv)
    lam1 = np.min(ritzv)
    if lowerb > upperb:
        raise ValueError("Bounds are incorrect")
    W = ch_filter(H, Vin, deg, lam1, lowerb, upperb)
    W, _ = scipy.linalg.qr(W, mode="economic", pivoting=False)
    V = H @ W
    G = _gram_upper(V, W)
    ritzv_raw, Q = scipy.linalg.eigh(G)
    order = np.argsort(ritzv_raw)
    return W @ Q[:, order], ritzv_raw[order]


def lanczos_krylov(B, v, m: int, nev: int, test: int, tol: float = 1e-5):
    """m-step Lanczos without reorthogonalisation that keeps its basis:
    Eigensolvers/lanczosForChsubsp.py:33-132 and lanczos.py:38-146.

    test 0: no convergence test (the reference's choice for n > 35000);
    test 1: lanczosForChsubsp.py:99-119, stop when |tr1 - tr0| < tol * tr0
            (no absolute value on the right, so a negative trace never stops);
    test 2: lanczos_gpu.py:128-137, |tr1 - tr0| < tol * |tr0| (the CPU
            lanczos.py:125-134 indexes an empty list there and cannot run).
    Traces are the sums of the nev lowest eigenvalues of T_k, taken at
    k >= min(8 nev, m) with k % 10 == 0 and at k = m.

    Returns (VV[:, :k], alpha[:k], beta[:k], k, rr, X): rr ascending
    eigenvalues of T_k and X its eigenvectors (scipy.linalg.eigh as the
    reference), beta[k-1] the residual norm of the last step."""
    n = B.shape[0]
    v1 = np.asarray(v, dtype=float).reshape(-1)
    v1 = v1 / np.linalg.norm(v1)
    v0 = np.zeros(n)
    bet = 0.0
    VV = np.zeros((n, m))
    alpha, beta = np.zeros(m), np.zeros(m)
    traces = []
    n_test = min(8 * nev, m)
    k = 0
    while k < m:
        VV[:, k] = v1
        w = B @ v1 - bet * v0
        alp = np.vdot(v1, w)
        w = w - alp * v1
        bet = np.linalg.norm(w)
        v0 = v1
        v1 = w * (1.0 / bet)
        alpha[k], beta[k] = alp, bet
        k += 1
        if test and ((k >= n_test and k % 10 == 0) or k == m):
            T = np.diag(alpha[:k]) + np.diag(beta[:k - 1], 1) + np.diag(beta[:k - 1], -1)
            traces.append(np.sum(np.sort(np.linalg.eigvalsh(T))[:nev]))
            if len(traces) > 1:
                lim = tol * traces[-2] if test == 1 else tol * abs(traces[-2])
                if abs(traces[-1] - traces[-2]) < lim:
                    break
    T = np.diag(alpha[:k]) + np.diag(beta[:k - 1], 1) + np.diag(beta[:k - 1], -1)
    rr, X = scipy.linalg.eigh(T)
    order = np.argsort(rr)
    return VV[:, :k], alpha[:k], beta[:k], k, rr[order], X[:, order]


def distinct_count(rr, gap: float = 1e-5) -> int:
    """Number of values left after the reference's near-duplicate pruning of
    the ascending Ritz values (lanczosForChsubsp.py:148-154, lanczos.py:165-174):
    walking upwards, a value within `gap` of the last kept one is dropped."""
    rr = np.asarray(rr)
    if rr.size == 0:
        return 0
    kept, anchor = 1, rr[0]
    for x in rr[1:]:
        if abs(anchor - x) >= gap:
            kept += 1
            anchor = x
    return kept


def ghost_width(nev: int, rr, k: int) -> int:
    """mev = int(min(nev * min(1.8 ** (len(rr)/distinct), 3.2), k)):
    lanczosForChsubsp.py:156-157, lanczos.py:177-179."""
    mult = min(1.8 ** (len(rr) / distinct_count(rr)), 3.2)
    return int(min(nev * mult, k))


def _krylov_ritz(B, VV, X, mev, nev):
    """W = VV X[:, :mev], Householder QR, Rayleigh-Ritz (upper triangle
    mirrored), the nev lowest pairs: lanczosForChsubsp.py:159-190 and
    lanczos.py:182-221."""
    W = VV @ X[:, :mev]
    W, _ = scipy.linalg.qr(W, mode="economic", pivoting=False)
    G = _gram_upper(B @ W, W)
    rr, Q = scipy.linalg.eigh(G)
    order = np.argsort(rr)
    return W @ Q[:, order[:nev]], rr[order][:nev]


def lanczos_for_chsubsp(B, nev: int, v, m: int):
    """Eigensolvers/lanczosForChsubsp.py:7-193 (reorth = 0): returns
    (W n x nev, lam[nev], bound) with bound = max|theta| + beta_k."""
    n = B.shape[0]
    VV, _, beta, k, rr, X = lanczos_krylov(B, v, m, nev, 0 if n > 35000 else 1)
    bound = float(np.max(np.abs(rr)) + beta[k - 1])
    W, lam = _krylov_ritz(B, VV, X, ghost_width(nev, rr, k), nev)
    return W, lam, bound


def chsubsp(deg: int, nev: int, H):
    """Chebyshev subspace iteration from a Lanczos start,
    Eigensolvers/chsubsp.py:10-91: Lanczos with max(3 nev, 450) steps, then
    at most 30 rounds of scaled filter + QR + Rayleigh-Ritz until the Ritz
    trace moves by less than 5 %."""
    n = H.shape[0]
    W, ritzv, upperb = lanczos_for_chsubsp(H, nev, np.random.randn(n), max(3 * nev, 450))
    tr0 = np.sum(ritzv)
    for _ in range(30):
        lam1, lowerb = np.min(ritzv), np.max(ritzv)
        if lowerb > upperb:
            raise ValueError("bounds are wrong")
        W = ch_filter(H, W, deg, lam1, lowerb, upperb)
        W, _ = scipy.linalg.qr(W, mode="economic", pivoting=False)
        G = _gram_upper(H @ W, W)
        ritzv, Q = scipy.linalg.eigh(G)
        W = W @ Q
        tr1 = np.sum(ritzv[:nev])
        if abs(tr1 - tr0) < 0.05 * abs(tr1):
            break
        tr0 = tr1
    return W, ritzv


def lanczos(B, nev: int, v, m: int, tol: float = 1e-5):
    """Eigensolvers/lanczos.py:10-223 (reorth = 0, no polynomial filtering),
    with the convergence test of its GPU twin (lanczos_gpu.py:128-137) for
    n <= 35000.  Returns (W n x nev, lam[nev])."""
    n = B.shape[0]
    VV, _, _, k, rr, X = lanczos_krylov(B, v, m, nev, 0 if n > 35000 else 2, tol)
    return _krylov_ritz(B, VV, X, ghost_width(nev, rr, k), nev)


def fermi_dirac(lam, ef, temp, nelec):
    """Eigensolvers/FermiDirac.py:3-31 (kT = T * 6.33327186e-06, spin 1)."""
    kT = temp * 6.33327186e-06
    logits = (lam - ef) / kT
    e = np.exp(-np.abs(logits))
    occ = np.where(logits >= 0, e / (1.0 + e), 1.0 / (1.0 + e))
    return np.sum(occ) - nelec / 2, occ


def occupations(lam, temp, nelec, tol):
    """Bisection for the Fermi level, Eigensolvers/occupations.py:5-56."""
    lam = np.asarray(lam, dtype=np.float64)
    its = 0
    a = np.min(lam) - 1
    fa, _ = fermi_dirac(lam, a, temp, nelec)
    lmax = min(max(1, int(np.ceil(nelec / 2)) + 1), len(lam))
    b = lam[lmax - 1] + 1
    fb, _ = fermi_dirac(lam, b, temp, nelec)
    c = (b + a) / 2
    fc, occ = fermi_dirac(lam, c, temp, nelec)
    error = 2 * np.sum(occ) - nelec
    if fa * fb > tol:
        return b, np.ones(len(lam))
    while abs(error) > tol and its < 200:
        its += 1
        c = (b + a) / 2
        fc, occ = fermi_dirac(lam, c, temp, nelec)
        error = 2 * np.sum(occ) - nelec
        if fc * fb < 0:
            a = c
        else:
            b = c
            fb = fc
    return c, occ


def pcg(A, rhs, x0, m, tol):
    """Unpreconditioned CG, Eigensolvers/pcg.py:7-85.  In the reference the
    first search direction p aliases the residual array r (z = r; p = z), so
    the in-place update r -= alp*Ap also moves p, and the first direction
    update gives p = (1 + beta) * r_1.  That is kept here."""
    x = np.array(x0, dtype=np.float64)
    r = rhs - A.dot(x)
    ro1 = np.dot(r, r)
    tol1 = tol * tol * ro1
    its = 0
    p = None
    while its < m and ro1 > tol1:
        its += 1
        ro = ro1
        ap = A.dot(r if p is None else p)
        alp = ro / np.dot(ap, r if p is None else p)
        x += alp * (r if p is None else p)
        r = r - alp * ap
        ro1 = np.dot(r, r)
        bet = ro1 / ro
        p = r + bet * r if p is None else r + bet * p
    return x, its


def pcg_prec(A, rhs, x0, m, tol, prec):
    """The preconditioned branch of Eigensolvers/pcg.py:7-85: z = M r,
    p = z (a fresh array, so no aliasing), ro1 = z.r, stop when
    ro1 <= tol^2 z0.r0; each step x += alp p, r -= alp Ap, z = M r,
    ro1 = z.r, p = z + (ro1/ro) p."""
    x = np.array(x0, dtype=np.float64)
    r = rhs - A.dot(x)
    z = prec(r)
    p = z
    ro1 = np.dot(z, r)
    tol1 = tol * tol * ro1
    its = 0
    while its < m and ro1 > tol1:
        its += 1
        ro = ro1
        ap = A.dot(p)
        alp = ro / np.dot(ap, p)
        x += alp * p
        r = r - alp * ap
        z = prec(r)
        ro1 = np.dot(z, r)
        p = z + (ro1 / ro) * p
    return x, its


def spectral_preconditioner(domain: dict, order: int):
    """M = S Lambda^-1 S with S the orthonormal 3-D DST-I of the box and
    Lambda the FD stencil's symbol at the DST frequencies: the exact inverse
    of the stencil continued by odd reflection across the faces (the GPU's
    cg_prec = 1 preconditioner; the reference's own cg_prec path cannot run,
    see pcg_spectral.cu).  Returns r -> M r on flat x-fastest vectors."""
    import scipy.fft

    nx, ny, nz, h = domain["nx"], domain["ny"], domain["nz"], domain["h"]
    c0, cs = fd_stencil(order)

    def lam(m):
        th = np.pi * np.arange(1, m + 1) / (m + 1)
        v = np.full(m, c0 / 3.0)
        for d, c in enumerate(cs, start=1):
            v += 2.0 * c * np.cos(d * th)
        return v / (h * h)

    L = lam(nz)[:, None, None] + lam(ny)[None, :, None] + lam(nx)[None, None, :]

    def apply(r):
        u = np.asarray(r, dtype=np.float64).reshape(nz, ny, nx)
        s = scipy.fft.dstn(u, type=1, norm="ortho")
        return scipy.fft.idstn(s / L, type=1, norm="ortho").ravel()

    return apply


# ----------------------------------------------------------------------------
# mixers (Mixer/msecant1.py, Mixer/msecant2.py with Mixer/includemix.py parameters)
# ----------------------------------------------------------------------------
def qinv(A, tol=np.finfo(float).eps):
    """Quasi-inverse by pivoted QR, Mixer/qinv.py:5-62."""
    m, n = A.shape
    if m < n:
        return qinv(A.T, tol).T
    tol = tol * np.linalg.norm(A, np.inf)
    Q, R, P = scipy.linalg.qr(A, mode="economic", pivoting=True)
    r = n
    for i in range(n):
        if abs(R[i, i]) < tol:
            r = i
            break
    S = np.zeros((r, r))
    for j in range(r - 1, -1, -1):
        S[j, j] = 1 / R[j, j]
        for i in range(j - 1, -1, -1):
            t = 0
            for kk in range(i + 1, r):
                t += R[i, kk] * S[kk, j]
            S[i, j] = -t / R[i, i]
    B = np.zeros((n, m))
    B[:r, :] = S @ Q[:, :r].T
    q = np.zeros(n, dtype=int)
    for i in range(n):
        q[P[i]] = i
    return B[q, :]


class MSecant1:
    """Multisecant Type-I (Broyden-1 with group_size 1, mix 0.5, restart
    factor 0.1), Mixer/msecant1.py:6-175 with Mixer/includemix.py:21-49."""

    def __init__(self, mix=0.5, group_size=1, restart_factor=0.1):
        self.mix, self.sz, self.rf = mix, group_size, restart_factor
        self.tol = np.finfo(float).eps
        self.DX = None
        self.DF = None
        self.N = None

    def __call__(self, x1, f1):
        mix, sz = self.mix, self.sz
        x1 = np.asarray(x1, dtype=np.float64).ravel()
        f1 = np.asarray(f1, dtype=np.float64).ravel()
        m = 0 if self.DX is None else self.DX.shape[1]
        if m == 0:
            self.DX = x1[:, None].copy()
            self.DF = f1[:, None].copy()
            return x1 + mix * f1, 0
        if m >= 2:
            if np.linalg.norm(self.DF[:, m - 1]) < self.rf * np.linalg.norm(f1):
                xr = self.DX[:, m - 1].copy()
                fr = self.DF[:, m - 1].copy()
                self.DX = xr[:, None]
                self.DF = fr[:, None]
                self.N = None
                return xr + mix * fr, 0
        res = (m + sz - 1) % sz + 1
        ngroup = (m - res) // sz
        self.DX[:, m - 1] = x1 - self.DX[:, m - 1]
        self.DF[:, m - 1] = f1 - self.DF[:, m - 1]
        dx = self.DX[:, m - 1].copy()
        self.DX[:, m - 1] = self.DX[:, m - 1] + mix * self.DF[:, m - 1]
        for i in range(1, ngroup + 1):
            s, e = (i - 1) * sz, i * sz
            self.DX[:, m - 1] = self.DX[:, m - 1] - self.DX[:, s:e] @ (self.DF[:, s:e].T @ self.DF[:, m - 1])
        x_new = x1 + mix * f1
        for i in range(1, ngroup + 1):
            s, e = (i - 1) * sz, i * sz
            x_new = x_new - self.DX[:, s:e] @ (self.DF[:, s:e].T @ f1)
        if self.N is None or self.N.shape[1] < res:
            self.N = np.zeros((x1.size, sz))
        self.N[:, res - 1] = -mix * dx
        for i in range(1, ngroup + 1):
            s, e = (i - 1) * sz, i * sz
            self.N[:, res - 1] = self.N[:, res - 1] + self.DF[:, s:e] @ (self.DX[:, s:e].T @ dx)
        M = self.N[:, :res].T @ self.DF[:, m - res:m]
        C = qinv(M, self.tol)
        if res == sz:
            self.DF[:, m - sz:m] = self.N[:, :sz] @ C.T
            x_new = x_new - self.DX[:, m - res:m] @ (self.DF[:, m - res:m].T @ f1)
        else:
            x_new = x_new - self.DX[:, m - res:m] @ ((C @ self.N[:, :res].T) @ f1)
        self.DX = np.hstack([self.DX, x1[:, None]])
        self.DF = np.hstack([self.DF, f1[:, None]])
        return x_new, m


class MSecant2:
    """Multisecant Type-II update, Mixer/msecant2.py:6-100 with the parameters
    of Mixer/includemix.py:21-49 (mix 0.5, restart factor 0.1, EN_like 0);
    group_size 0 takes all iterates as one group: Anderson mixing.  A restart
    sets the EN stage to 2 whatever EN_like is (msecant2.py:45-51), after
    which the stage alternates 2 -> 1 -> 2: on stage-1 calls the newest
    difference is not formed and, with a full last group, the stored DF C is
    used as it is; on stage-2 calls the new iterate is not appended."""

    def __init__(self, mix=0.5, group_size=0, restart_factor=0.1, en_like=0):
        self.mix, self.gs, self.rf, self.en_like = mix, group_size, restart_factor, en_like
        self.tol = np.finfo(float).eps
        self.DX = None
        self.DF = None
        self.en = None

    def __call__(self, x1, f1):
        mix = self.mix
        x1 = np.asarray(x1, dtype=np.float64).ravel()
        f1 = np.asarray(f1, dtype=np.float64).ravel()
        if self.DX is None:
            self.DX = x1[:, None].copy()
            self.DF = f1[:, None].copy()
            self.en = 0 if self.en_like == 0 else 2
            return x1 + mix * f1, 0
        m = self.DX.shape[1]
        sz = m + 1 if self.gs == 0 else self.gs
        if self.en != 1 and m >= 2 and np.linalg.norm(self.DF[:, -1], 2) < self.rf * np.linalg.norm(f1, 2):
            self.DX = x1[:, None].copy()
            self.DF = f1[:, None].copy()
            self.en = 2
            return x1 + mix * f1, 0
        res = (m + sz - 1) % sz + 1
        ngroup = (m - res) // sz
        if self.en != 1:
            self.DX[:, m - 1] = x1 - self.DX[:, m - 1]
            self.DF[:, m - 1] = f1 - self.DF[:, m - 1]
            self.DX[:, m - 1] += mix * self.DF[:, m - 1]
            for i in range(ngroup):
                s, e = i * sz, (i + 1) * sz
                self.DX[:, m - 1] -= self.DX[:, s:e] @ (self.DF[:, s:e].T @ self.DF[:, m - 1])
        x_new = x1 + mix * f1
        for i in range(ngroup):
            s, e = i * sz, (i + 1) * sz
            x_new -= self.DX[:, s:e] @ (self.DF[:, s:e].T @ f1)
        if self.en == 1 and res == sz:
            x_new -= self.DX[:, ngroup * sz:m] @ (self.DF[:, ngroup * sz:m].T @ f1)
        else:
            C2 = qinv(self.DF[:, m - res:m], self.tol)
            C = C2 @ C2.T
            if res == sz:
                self.DF[:, m - sz:m] = self.DF[:, m - sz:m] @ C
                x_new -= self.DX[:, m - res:m] @ (self.DF[:, m - res:m].T @ f1)
            else:
                x_new -= self.DX[:, m - res:m] @ ((self.DF[:, m - res:m] @ C).T @ f1)
        if self.en != 2:
            self.DX = np.hstack([self.DX, x1[:, None]])
            self.DF = np.hstack([self.DF, f1[:, None]])
        if self.en == 1:
            self.en = 2
        elif self.en == 2:
            self.en = 1
        return x_new, m


# ----------------------------------------------------------------------------
# energies and the SCF loop (rsdft_solver.py)
# ----------------------------------------------------------------------------
def energy_components(rho, hpot, hpot0, vxc, exc, lam, occ, nev, e_nuc, h):
    """rsdft_solver.py:128-153 (Rydberg)."""
    esum = float(np.sum(lam[:nev] * occ[:nev]))
    eig = 4.0 * esum
    eh = float(np.sum(rho * (hpot + hpot0)) * h ** 3)
    vxc_sum = float(np.sum(rho * vxc) * h ** 3)
    total = eig - eh + float(exc) - vxc_sum + float(e_nuc)
    return {"eigen_sum_ry": eig, "hartree_ry": eh, "xc_ry": float(exc), "ion_ry": float(e_nuc),
            "total_ry": total}


def build_system(atoms: list, *, h: float, radius: float, elements: dict | None = None):
    """Domain for a given spacing and sphere radius (bohr), as
    rsdft_setup.estimate_radius_and_grid (rsdft_setup.py:133-150) does with a
    radius override."""
    nx = int(2 * radius / h) + 1
    nx = 2 * ((nx + 1) // 2)
    rad = 0.5 * h * (nx - 1)
    return {"radius": rad, "nx": nx, "ny": nx, "nz": nx, "h": h}


class OracleSCF:
    """The SCF of rsdft_solver.run_rsdft_calculation (rsdft_solver.py:156-462)
    for density_method = sad, adaptive_scheme = 0, cg_prec = 0 or 1 (the
    spectral preconditioner), any diagmeth
    (rsdft_solver.py:287-317: 3 first_filt, 2 chsubsp, 0 lanczos, then chefsi1;
    1 lanczos at every iteration),
    split into setup() and step() so that a bounded number of iterations can
    be timed.  Wall times (s) are kept in t_setup and in each history entry."""

    def __init__(self, domain: dict, atoms: list, *, nev: int, poldeg: int = 10, tol: float = 2e-4,
                 maxits: int = 40, fd_order: int = 8, fermi_temp: float = 500.0, z_charge: float = 0.0,
                 elements=None, tables=None, diagmeth: int = 3, density_method: str = "sad", density=None,
                 operator: str = "csr", cg_prec: int = 0):
        if operator not in ("csr", "stencil"):
            raise ValueError(f"operator must be 'csr' or 'stencil', not {operator!r}")
        self.domain, self.atoms, self.nev, self.poldeg, self.tol = domain, atoms, nev, poldeg, tol
        self.operator = operator
        self.cg_prec = cg_prec
        self.diagmeth = diagmeth
        self.density_method, self.density = density_method, density
        self.maxits, self.fd_order, self.fermi_temp, self.z_charge = maxits, fd_order, fermi_temp, z_charge
        self.elements = elements or load_elements()
        self.tables = tables or load_tables()
        self.history: list = []
        self.its = 0
        self.t_setup = None

    def setup(self) -> None:
        import time

        t0 = time.perf_counter()
        d, h = self.domain, self.domain["h"]
        self.A = laplacian(d, self.fd_order) if self.operator == "csr" else StencilLaplacian(d, self.fd_order)
        n = self.n = self.A.shape[0]
        self.Hpot = np.zeros(n)
        self.err = 10.0 + self.tol
        self.e_nuc = nuclear(self.atoms, self.elements)
        dm = self.density_method
        if dm == "ml":   # rsdft_solver.py:96-108: the file density becomes the reference charge
            self.rho0, self.hpot0, self.ppot, self.info = ml_density_start(d, self.atoms, self.elements,
                                                                           self.tables, self.density,
                                                                           self.fd_order)
        else:
            self.rho0, self.hpot0, self.ppot, self.info = pseudo_diag(ml_grid(d) if dm == "sad_ml_grid" else d,
                                                                      self.atoms, self.elements, self.tables)
        projs = projectors(ml_grid(d) if dm in ("ml", "sad_ml_grid") else d, self.atoms, self.elements,
                           self.tables)
        self.projs = projs
        vnl = nonlocal_csr(projs, n) if self.operator == "csr" else None
        xcpot, self.exc = exc_nspn(h, self.rho0 / h ** 3)
        self.XCpot = xcpot
        self.nelec = nelectrons(self.atoms, self.elements) - self.z_charge
        self.pot = self.ppot + self.hpot0 + 0.5 * xcpot
        self.mixer = MSecant1()
        self.half_a_plus_vnl = 0.5 * self.A + vnl if self.operator == "csr" else None
        self.W = self.lam = None
        self.rho = np.zeros(n)
        self.t_setup = time.perf_counter() - t0

    def done(self) -> bool:
        return not (self.err > self.tol and self.its < self.maxits)

    def step(self) -> dict:
        import time

        t0 = time.perf_counter()
        n, h, nev = self.n, self.domain["h"], self.nev
        self.its += 1
        if self.operator == "csr":
            B = (self.half_a_plus_vnl + sp.diags(self.pot, 0, shape=(n, n))).tocsr()
        else:
            B = StencilHamiltonian(self.domain, self.fd_order, self.projs, self.pot)
        dm = self.diagmeth
        if dm == 1 or (self.its == 1 and dm == 0):
            # rsdft_solver.py:63-68 (CPU vector) and :47-49 (nev + 500 steps)
            self.W, self.lam = lanczos(B, nev + 15, np.random.randn(n, 1), nev + 500, 1e-5)
        elif self.its == 1 and dm == 2:
            self.W, self.lam = chsubsp(self.poldeg, nev + 15, B)
        elif self.its == 1:
            self.W, self.lam = first_filt(nev + 15, B, self.poldeg)
        else:
            self.W, self.lam = chefsi1(self.W, self.lam, self.poldeg, nev, B)
        _, occ = occupations(self.lam[:nev], self.fermi_temp, self.nelec, 1e-6)
        rho = (self.W[:, :nev] ** 2) @ (2 * occ)
        hrhs = (4 * np.pi / h ** 3) * (rho - self.rho0)
        self.rho = rho / h ** 3
        if self.cg_prec:
            # rsdft_solver.py:336-342 with the preconditioned branch of pcg.py;
            # the preconditioner is the spectral inverse of the stencil (the
            # reference's own ILU path cannot run, see pcg_prec)
            if getattr(self, "_prec", None) is None:
                self._prec = spectral_preconditioner(self.domain, self.fd_order)
            self.Hpot, cg_its = pcg_prec(self.A, hrhs, self.Hpot, 200, 1e-5, self._prec)
        else:
            self.Hpot, cg_its = pcg(self.A, hrhs, self.Hpot, 200, 1e-5)
        self.XCpot, self.exc = exc_nspn(h, self.rho)
        pot_new = self.ppot + 0.5 * self.XCpot + self.Hpot + self.hpot0
        self.err = float(np.linalg.norm(pot_new - self.pot) / np.linalg.norm(pot_new))
        en = energy_components(self.rho, self.Hpot, self.hpot0, self.XCpot, self.exc, self.lam, occ, nev,
                               self.e_nuc, h)
        self.occ = occ
        self.pot, _ = self.mixer(self.pot, pot_new - self.pot)
        rec = {"iter": self.its, "err": self.err, "lam": self.lam.copy(), "occ": np.asarray(occ).copy(),
               "cg_its": cg_its, "wall": time.perf_counter() - t0, **en}
        self.history.append(rec)
        return rec

    def result(self) -> dict:
        return {"rho": self.rho, "hpot": self.Hpot, "xc_potential": self.XCpot, "exc": float(self.exc),
                "potential": self.pot, "W": self.W, "eigenvalues": self.lam, "occupations": self.occ,
                "iterations": self.its, "error": self.err, "converged": self.err <= self.tol,
                "e_nuc0": self.e_nuc, "hpot0": self.hpot0, "rho0": self.rho0, "ppot": self.ppot,
                "history": self.history, "energies": self.history[-1] if self.history else None,
                "diag_info": self.info, "t_setup": self.t_setup}


def run_scf(domain: dict, atoms: list, *, nev: int, poldeg: int = 10, tol: float = 2e-4,
            maxits: int = 40, fd_order: int = 8, fermi_temp: float = 500.0, seed: int | None = None,
            z_charge: float = 0.0, elements=None, tables=None, log=None, diagmeth: int = 3,
            density_method: str = "sad", density=None, operator: str = "csr") -> dict:
    """Run OracleSCF to convergence; with a seed, numpy's global generator is
    seeded first so the random draws match a reference run with that seed."""
    if seed is not None:
        np.random.seed(seed)
    scf = OracleSCF(domain, atoms, nev=nev, poldeg=poldeg, tol=tol, maxits=maxits, fd_order=fd_order,
                    fermi_temp=fermi_temp, z_charge=z_charge, elements=elements, tables=tables, diagmeth=diagmeth,
                    density_method=density_method, density=density, operator=operator)
    scf.setup()
    while not scf.done():
        rec = scf.step()
        if log:
            log(f"iter {rec['iter']} err {rec['err']:.3e} E {rec['total_ry']:.10f}")
    return scf.result()
