"""Device-side objects and solver stages over libpsc.

Vectors are torch CUDA tensors used only as device memory; every
computation is a libpsc kernel.  A block of k vectors is a (k, n) tensor,
i.e. an n x k column-major matrix with leading dimension n, which is the
layout the C ABI expects.

The stages mirror the reference's backend functions
(PARSEC.py src/Eigensolvers, src/V_ion, src/V_xc, src/Mixer) with the same
argument meaning; results stay on the device (as the reference's CuPy path
returns CuPy arrays) and the caller converts what it logs.
"""
from __future__ import annotations

import ctypes
import itertools
import math
from ctypes import byref, c_int, c_long, c_void_p

import numpy as np
import torch

from . import _lib
from ._lib import F32, F64, PscError, call

_DT = {F64: torch.float64, F32: torch.float32}


def _p(t: torch.Tensor | None) -> c_void_p:
    return c_void_p(t.data_ptr() if t is not None else None)


def _stream() -> c_void_p:
    return c_void_p(torch.cuda.current_stream().cuda_stream)


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise PscError("the GPU backend needs a CUDA device (no CPU fallback exists)")
    _lib.load()
    return torch.device("cuda", torch.cuda.current_device())


class GridContext:
    """libpsc context of one cube domain and finite-difference order."""

    def __init__(self, domain: dict, fd_order: int = 8, seed: int = 0):
        self.device = require_cuda()
        self.nx, self.ny, self.nz = int(domain["nx"]), int(domain["ny"]), int(domain["nz"])
        self.h = float(domain["h"])
        self.radius = float(domain["radius"])
        self.fd_order = int(fd_order)
        self.n = self.nx * self.ny * self.nz
        ptr = c_void_p()
        call("psc_ctx_create", self.nx, self.ny, self.nz, self.h, self.fd_order, byref(ptr))
        self.ptr = ptr
        self.species: dict[str, int] = {}
        self._seed = itertools.count(int(seed) * 1_000_003 + 17)
        self.projectors = None
        self.mask_radius = 0.0

    def __del__(self):
        try:
            if getattr(self, "ptr", None) and self.ptr.value:
                _lib.load().psc_ctx_destroy(self.ptr)
                self.ptr = c_void_p()
        except Exception:
            pass

    def matches(self, domain: dict, fd_order: int) -> bool:
        return (self.nx, self.ny, self.nz, self.h, self.radius, self.fd_order) == (
            int(domain["nx"]), int(domain["ny"]), int(domain["nz"]), float(domain["h"]), float(domain["radius"]),
            int(fd_order))

    def call(self, name: str, *args) -> None:
        call(name, self.ptr, *args, ctx=self.ptr)

    def set_sphere_mask(self, radius: float) -> None:
        """H X is zero outside the sphere of this radius (bohr) around the
        cube's centre; 0 restores the cube (psc_set_sphere_mask)."""
        self.call("psc_set_sphere_mask", float(radius), _stream())
        self.mask_radius = float(radius) if radius > 0 else 0.0

    def mask_block(self, X: torch.Tensor) -> torch.Tensor:
        """Zero X (a (k, n) block or an n-vector) outside the sphere mask, in place."""
        if self.mask_radius > 0:
            k = 1 if X.dim() == 1 else X.shape[0]
            self.call("psc_mask_block", _dtype_code(X), _p(X), self.n, k, _stream())
        return X

    def inside_count(self) -> int:
        """Grid points the Hamiltonian produces: inside the sphere mask, or all."""
        if self.mask_radius <= 0:
            return self.n
        c = 0.5 * self.h * (np.array([self.nx, self.ny, self.nz]) - 1)
        x = np.arange(self.nx) * self.h - c[0]
        y = np.arange(self.ny) * self.h - c[1]
        z = np.arange(self.nz) * self.h - c[2]
        d2 = (z[:, None, None] ** 2 + y[None, :, None] ** 2) + x[None, None, :] ** 2
        return int(np.count_nonzero(d2 <= self.mask_radius ** 2))

    def next_seed(self) -> int:
        return next(self._seed)

    def empty(self, *shape, dtype=torch.float64) -> torch.Tensor:
        return torch.empty(*shape, dtype=dtype, device=self.device)

    def zeros(self, *shape, dtype=torch.float64) -> torch.Tensor:
        return torch.zeros(*shape, dtype=dtype, device=self.device)

    def register_species(self, symbol: str, elem, tables) -> int:
        if symbol in self.species:
            return self.species[symbol]
        sid = len(self.species)
        tab = np.ascontiguousarray(tables[symbol], dtype=np.float64)
        row = elem[symbol]
        self.call("psc_set_species", sid, tab.shape[0], tab.ctypes.data_as(c_void_p), float(row["Zvalue"]),
                  float(row["R"]))
        self.species[symbol] = sid
        return sid

    def atom_arrays(self, atoms, elem, tables):
        sp, xyz = [], []
        for a in atoms:
            sid = self.register_species(a["typ"], elem, tables)
            c = np.asarray(a["coord"], dtype=np.float64).reshape(-1, 3)
            for row in c:
                sp.append(sid)
                xyz.append(row)
        return (np.ascontiguousarray(sp, dtype=np.int32), np.ascontiguousarray(np.array(xyz, dtype=np.float64)))

    def status(self, clear: bool = True) -> list[int]:
        flags = (c_int * 8)()
        self.call("psc_status", flags, int(clear), _stream())
        return list(flags)

    def check_status(self) -> None:
        f = self.status(clear=True)
        if f[0]:
            raise ValueError("Bounds are incorrect")
        if f[1]:
            raise PscError(f"Cholesky of the overlap matrix failed at column {f[1] - 1} (subspace rank deficient)")
        if f[3]:
            raise PscError("TMA stencil pipeline wait timed out")
        if f[4]:
            raise PscError("persistent CG grid barrier timed out")
        if f[5]:
            raise PscError("tensor-core Gram pipeline wait timed out")
        if f[6]:
            raise PscError("tensor-core block product pipeline wait timed out")
        if f[7]:
            raise PscError("tensor-core conv3d pipeline wait timed out")

    def info(self) -> dict:
        out = (c_long * 8)()
        self.call("psc_ctx_info", out)
        keys = ("nx", "ny", "nz", "n", "nl_atoms", "nl_points", "nl_touched", "stencil_radius")
        return dict(zip(keys, list(out)))


class NonlocalProjectors:
    """Factored Kleinman-Bylander term held by the context (what the
    reference's pseudoNL returns as an n x n sparse matrix)."""

    def __init__(self, ctx: GridContext):
        self.ctx = ctx
        self.shape = (ctx.n, ctx.n)
        i = ctx.info()
        self.n_atoms, self.n_points, self.n_touched = i["nl_atoms"], i["nl_points"], i["nl_touched"]

    def tables(self):
        """(atom_off, idx, u[3, points], w) on the host."""
        na, npt = self.n_atoms, self.n_points
        off = np.zeros(na + 1, dtype=np.int32)
        idx = np.zeros(npt, dtype=np.int32)
        u = np.zeros(3 * npt, dtype=np.float64)
        w = np.zeros(na, dtype=np.float64)
        if na:
            self.ctx.call("psc_projector_export", off.ctypes.data_as(c_void_p), idx.ctypes.data_as(c_void_p),
                          u.ctypes.data_as(c_void_p), w.ctypes.data_as(c_void_p))
        return off, idx, u.reshape(3, npt), w


class Laplacian:
    """A = -Lap_h (rsdft_solver.py:186), applied by the stencil kernel."""

    def __init__(self, ctx: GridContext):
        self.ctx = ctx
        self.shape = (ctx.n, ctx.n)

    def __matmul__(self, x: torch.Tensor) -> torch.Tensor:
        x = x.contiguous()
        k = 1 if x.dim() == 1 else x.shape[0]
        y = torch.empty_like(x)
        self.ctx.call("psc_laplacian_apply", _p(x), _p(y), k, self.ctx.n, _stream())
        return y


class Hamiltonian:
    """H = 0.5 A + V_nl + diag(pot) (rsdft_solver.py:263,285), matrix-free.
    `dtype` selects the precision of H.X (F64 or F32 blocks)."""

    def __init__(self, ctx: GridContext, pot: torch.Tensor, dtype: int = F64):
        self.ctx = ctx
        self.shape = (ctx.n, ctx.n)
        self.dtype = dtype
        self.set_potential(pot)

    def set_potential(self, pot: torch.Tensor) -> None:
        self.pot = pot
        self.ctx.call("psc_set_potential", _p(pot), _stream())

    def __matmul__(self, X: torch.Tensor) -> torch.Tensor:
        X = X.contiguous()
        k = 1 if X.dim() == 1 else X.shape[0]
        dt = F32 if X.dtype == torch.float32 else F64
        Y = torch.empty_like(X)
        self.ctx.call("psc_apply_h", dt, _p(X), self.ctx.n, _p(Y), self.ctx.n, k, _stream())
        return Y


def _dtype_code(t: torch.Tensor) -> int:
    return F32 if t.dtype == torch.float32 else F64


# ---------------------------------------------------------------------------
# eigensolver stages
# ---------------------------------------------------------------------------
def cheb_filter(H: Hamiltonian, W: torch.Tensor, T: torch.Tensor, deg: int, bounds: torch.Tensor, mode: int):
    """Filter W in place of (W, T); returns (result, other)."""
    which = c_int()
    H.ctx.call("psc_cheb_filter", _dtype_code(W), mode, deg, _p(bounds), _p(W), _p(T), H.ctx.n, W.shape[0],
               byref(which), _stream())
    return (T, W) if which.value else (W, T)


def orthonormalize(ctx: GridContext, W: torch.Tensor, T: torch.Tensor, passes: int = 2):
    which = c_int()
    ctx.call("psc_orthonormalize", _dtype_code(W), _p(W), _p(T), ctx.n, W.shape[0], passes, byref(which), _stream())
    return (T, W) if which.value else (W, T)


def rayleigh_ritz(ctx: GridContext, W: torch.Tensor, V: torch.Tensor, ritz: torch.Tensor):
    ctx.call("psc_rayleigh_ritz", _dtype_code(W), _p(W), _p(V), ctx.n, W.shape[0], _p(ritz), _stream())
    return V, W


def subspace_rr(ctx: GridContext, W: torch.Tensor, V: torch.Tensor, ritz: torch.Tensor):
    """Orthonormalise + Rayleigh-Ritz in one pass (psc_subspace_rr); result in V."""
    ctx.call("psc_subspace_rr", _dtype_code(W), _p(W), _p(V), ctx.n, W.shape[0], _p(ritz), _stream())
    return V, W


def lanczos_bound(ctx: GridContext, mode: int) -> torch.Tensor:
    out = ctx.empty(8)
    ctx.call("psc_lanczos_bound", mode, ctx.next_seed(), _p(out), _stream())
    return out


def first_filt(nev: int, H: Hamiltonian, polm: int = 10, dtype=torch.float64, log_trace=None,
               energ_tol: float = 0.08, max_iter: int | None = None):
    """First SCF step (Eigensolvers/first_filt.py:6-75): Lanczos bounds,
    random block, up to max_iter rounds of slim filter + orthonormalisation +
    Rayleigh-Ritz, stop when the Ritz trace moves by <= energ_tol (8 % and
    max(min(60 / polm, 5), 3) rounds in the reference; a start whose
    potential is already close to self-consistent, such as the learned one,
    can ask for a converged first subspace instead)."""
    ctx = H.ctx
    if polm < 10 or polm > 15:
        polm = 10
    if not max_iter:
        max_iter = max(min(int(60 / polm), 5), 3)
    lz = lanczos_bound(ctx, 0)                       # [uppbnd, ritz_0..5]
    bounds = ctx.empty(3)
    ctx.call("psc_filter_bounds", 1, _p(lz[1:7]), 6, _p(lz[0:1]), _p(bounds), _stream())
    W = ctx.empty(nev, ctx.n, dtype=dtype)
    ctx.call("psc_random", _dtype_code(W), 0, ctx.next_seed(), _p(W), ctx.n, ctx.n, nev, _stream())
    ctx.mask_block(W)
    T = torch.empty_like(W)
    ritz = ctx.empty(nev)
    tr0 = None
    for it in range(1, max_iter + 1):
        W, T = cheb_filter(H, W, T, polm, bounds, mode=1)
        W, T = subspace_rr(ctx, W, T, ritz)
        ctx.call("psc_filter_bounds", 2, _p(ritz), nev, _p(lz[0:1]), _p(bounds), _stream())
        tr = float(np.sum(ritz.cpu().numpy()))
        if log_trace:
            log_trace(it, tr)
        if it == 1:
            tr0 = tr
        else:
            if abs(tr - tr0) <= energ_tol * abs(tr0):
                break
            tr0 = tr
    ctx.check_status()
    return W, ritz


def chefsi1(W: torch.Tensor, ritzv: torch.Tensor, deg: int, nev: int, H: Hamiltonian):
    """One Chebyshev-filtered subspace step (Eigensolvers/chefsi1.py:10-69)."""
    ctx = H.ctx
    k = W.shape[0]
    if nev >= k:
        raise ValueError("Vin should have more than nev columns")
    lz = lanczos_bound(ctx, 1)
    bounds = ctx.empty(3)
    ctx.call("psc_filter_bounds", 0, _p(ritzv), k, _p(lz[0:1]), _p(bounds), _stream())
    T = torch.empty_like(W)
    W, T = cheb_filter(H, W, T, deg, bounds, mode=0)
    ritz = ctx.empty(k)
    W, T = subspace_rr(ctx, W, T, ritz)
    return W, ritz


def _start_vector(ctx: GridContext, v) -> torch.Tensor | None:
    if v is None:
        return None
    if isinstance(v, torch.Tensor):
        t = v.reshape(-1).to(device=ctx.device, dtype=torch.float64)
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1))).to(ctx.device)
    if t.numel() != ctx.n:
        raise ValueError(f"start vector has {t.numel()} entries, expected {ctx.n}")
    return t.contiguous()


def distinct_count(rr: np.ndarray, gap: float = 1e-5) -> int:
    """Values left after the reference's near-duplicate pruning of the
    ascending Lanczos Ritz values (Eigensolvers/lanczosForChsubsp.py:148-154,
    lanczos.py:165-174): walking upwards, a value within `gap` of the last
    kept one is dropped."""
    if rr.size == 0:
        return 0
    kept, anchor = 1, rr[0]
    for x in rr[1:]:
        if abs(anchor - x) >= gap:
            kept += 1
            anchor = x
    return kept


def lanczos_krylov(H: Hamiltonian, nev: int, m: int, test: int, v=None, tol: float = 1e-5):
    """m Lanczos steps with the basis kept in VV ((m+1) x n rows = columns of
    an n x (m+1) block); Eigensolvers/lanczosForChsubsp.py:33-132 and
    lanczos.py:38-146.  test 0: none; 1: lanczosForChsubsp's stop rule
    |tr1 - tr0| < tol * tr0; 2: lanczos_gpu.py:128-137's |tr1 - tr0| < tol |tr0|,
    with traces of the nev lowest eigenvalues of T_k at k >= min(8 nev, m),
    k % 10 == 0, and at k = m.  Returns (VV, ab, k, rr) with rr on the host."""
    ctx = H.ctx
    n = ctx.n
    VV = ctx.empty(m + 1, n)
    ab = ctx.zeros(2 * m)
    evals = ctx.empty(m)
    v0 = _start_vector(ctx, v)
    if v0 is None and ctx.mask_radius > 0:
        # a start that vanishes outside the sphere keeps the Krylov basis there
        v0 = ctx.empty(n)
        ctx.call("psc_random", F64, 1, ctx.next_seed(), _p(v0), n, n, 1, _stream())
    if v0 is not None and ctx.mask_radius > 0:
        v0 = ctx.mask_block(v0.clone())
    seed = ctx.next_seed()
    if not test:
        ctx.call("psc_lanczos_run", _p(v0), seed, 0, m, _p(VV), n, _p(ab), _stream())
        k = m
    else:
        n_test = min(8 * nev, m)
        stops = sorted({c for c in range(10, m + 1, 10) if c >= n_test} | {m})
        traces, k = [], 0
        for c in stops:
            ctx.call("psc_lanczos_run", _p(v0), seed, k, c, _p(VV), n, _p(ab), _stream())
            k = c
            ctx.call("psc_tridiag_eig", _p(ab), k, 0, _p(evals), None, 0, _stream())
            traces.append(float(evals[:min(nev, k)].sum().item()))
            if len(traces) > 1:
                lim = tol * traces[-2] if test == 1 else tol * abs(traces[-2])
                if abs(traces[-1] - traces[-2]) < lim:
                    break
    ctx.call("psc_tridiag_eig", _p(ab), k, 0, _p(evals), None, 0, _stream())
    return VV, ab, k, evals[:k].cpu().numpy()


def _krylov_ritz(H: Hamiltonian, VV: torch.Tensor, ab: torch.Tensor, k: int, rr: np.ndarray, nev: int,
                 dtype=torch.float64):
    """W = VV X[:, :mev] with mev = int(min(nev * min(1.8 ** (k / distinct), 3.2), k)),
    orthonormalised (dependent columns dropped), Rayleigh-Ritz, the nev lowest
    pairs (lanczosForChsubsp.py:148-190, lanczos.py:164-221)."""
    ctx = H.ctx
    n = ctx.n
    mev = int(min(nev * min(1.8 ** (len(rr) / distinct_count(rr)), 3.2), k))
    evals = ctx.empty(k)
    X = ctx.empty(mev, k)                       # k x mev, column-major, ld k
    ctx.call("psc_tridiag_eig", _p(ab), k, mev, _p(evals), _p(X), k, _stream())
    W = ctx.empty(max(mev, nev), n)
    ctx.call("psc_gemm_nn", F64, _p(VV), n, k, _p(X), mev, _p(W), n, _stream())
    T = torch.empty_like(W)
    rank, which = c_int(), c_int()
    ctx.call("psc_orthonormalize_rank", F64, _p(W), _p(T), n, mev, 1e-10, byref(rank), byref(which), _stream())
    B, S = (T, W) if which.value else (W, T)
    r = rank.value
    if r < nev:
        # as many directions as the reference's QR returns: fresh random
        # columns after the kept ones, then the whole block orthonormalised
        ctx.call("psc_random", F64, 1, ctx.next_seed(), _p(B[r:]), n, n, nev - r, _stream())
        ctx.mask_block(B[r:nev])
        B, S = orthonormalize(ctx, B[:nev], S[:nev])
        r = nev
    V = S[:r]
    ritz = ctx.empty(r)
    ctx.call("psc_rayleigh_ritz", F64, _p(B[:r]), _p(V), n, r, _p(ritz), _stream())
    W = V[:nev].contiguous() if dtype == torch.float64 else V[:nev].to(dtype)
    return W, ritz[:nev].clone(), mev, r


def lanczos_for_chsubsp(H: Hamiltonian, nev: int, m: int, v=None, dtype=torch.float64):
    """Eigensolvers/lanczosForChsubsp.py:7-193: (W, lam, bound) with bound =
    max|theta| + beta_k of the Lanczos tridiagonal."""
    ctx = H.ctx
    VV, ab, k, rr = lanczos_krylov(H, nev, m, 0 if ctx.n > 35000 else 1, v)
    beta = float(ab[2 * k - 1].item())
    bound = float(np.max(np.abs(rr)) + beta)
    W, lam, _, _ = _krylov_ritz(H, VV, ab, k, rr, nev, dtype)
    del VV
    return W, lam, bound


def chsubsp(deg: int, nev: int, H: Hamiltonian, v=None, dtype=torch.float64, log_trace=None):
    """Chebyshev subspace iteration from a Lanczos start
    (Eigensolvers/chsubsp.py:10-91): Lanczos with max(3 nev, 450) steps, then
    at most 30 rounds of scaled filter + orthonormalisation + Rayleigh-Ritz
    until the Ritz trace moves by less than 5 %."""
    ctx = H.ctx
    W, ritzv, upperb = lanczos_for_chsubsp(H, nev, max(3 * nev, 450), v, dtype)
    up = torch.tensor([upperb], dtype=torch.float64).to(ctx.device)
    bounds = ctx.empty(3)
    T = torch.empty_like(W)
    k = W.shape[0]
    ritz_h = ritzv.cpu().numpy()
    tr0 = float(np.sum(ritz_h))
    for it in range(30):
        if np.max(ritz_h) > upperb:
            raise ValueError("bounds are wrong")
        ctx.call("psc_filter_bounds", 0, _p(ritzv), k, _p(up), _p(bounds), _stream())
        W, T = cheb_filter(H, W, T, deg, bounds, mode=0)
        ritzv = ctx.empty(k)
        W, T = subspace_rr(ctx, W, T, ritzv)
        ritz_h = ritzv.cpu().numpy()
        tr1 = float(np.sum(ritz_h[:nev]))
        if log_trace:
            log_trace(it + 1, tr1)
        if abs(tr1 - tr0) < 0.05 * abs(tr1):
            break
        tr0 = tr1
    ctx.check_status()
    return W, ritzv


def lanczos(H: Hamiltonian, nev: int, v=None, m: int | None = None, tol: float = 1e-5, dtype=torch.float64):
    """Eigensolvers/lanczos.py:10-223 (reorth = 0), convergence test as its
    GPU twin lanczos_gpu.py:128-137 for n <= 35000: (W, lam)."""
    ctx = H.ctx
    if m is None:
        raise ValueError("lanczos needs the number of steps m")
    VV, ab, k, rr = lanczos_krylov(H, nev, int(m), 0 if ctx.n > 35000 else 2, v, tol)
    W, lam, _, _ = _krylov_ritz(H, VV, ab, k, rr, nev, dtype)
    del VV
    ctx.check_status()
    return W, lam


def occupations(ctx: GridContext, lam: torch.Tensor, temp: float, nelec: float, tol: float):
    """Fermi level and occupations (Eigensolvers/occupations.py:5-56)."""
    lam = lam.contiguous()
    ef = ctx.empty(1)
    occ = ctx.empty(lam.shape[0])
    ctx.call("psc_occupations", _p(lam), lam.shape[0], float(temp), float(nelec), float(tol), _p(ef), _p(occ),
             _stream())
    return ef, occ


def density(ctx: GridContext, W: torch.Tensor, nev: int, occ: torch.Tensor, rho0: torch.Tensor):
    """(rho [e/bohr^3], hrhs) from the first nev columns (rsdft_solver.py:324-328)."""
    h = ctx.h
    rho = ctx.empty(ctx.n)
    hrhs = ctx.empty(ctx.n)
    ctx.call("psc_density", _dtype_code(W), _p(W), ctx.n, nev, _p(occ), _p(rho0), 4 * np.pi / h ** 3, h ** 3,
             _p(rho), _p(hrhs), _stream())
    return rho, hrhs


def pcg(A: Laplacian, rhs: torch.Tensor, x0: torch.Tensor, maxit: int, tol: float, *prec):
    """CG on A x = rhs from x0 (Eigensolvers/pcg.py:7-85); x0 is not modified.
    With the reference's (PRE, precfun) pair (cg_prec = 1) the solve is the
    preconditioned branch of pcg.py with the spectral preconditioner of
    psc_pcg_poisson_prec, whatever PRE holds."""
    x = x0.clone()
    its = c_int()
    entry = "psc_pcg_poisson_prec" if len(prec) >= 2 else "psc_pcg_poisson"
    A.ctx.call(entry, _p(rhs), _p(x), int(maxit), float(tol), byref(its), _stream())
    return x, its.value


def poisson_precond(ctx: GridContext, r: torch.Tensor) -> torch.Tensor:
    """z = M r, the cg_prec = 1 preconditioner (exact inverse of the FD stencil
    continued by odd reflection, by 3-D sine transforms)."""
    z = torch.empty_like(r)
    ctx.call("psc_poisson_precond", _p(r), _p(z), _stream())
    return z


def lda_xc(ctx: GridContext, rho: torch.Tensor):
    """LDA XC (V_xc/exc_nspn.py:8-103): (vxc [Ry], out=[exc, max rho, min rho]) on the device."""
    vxc = ctx.empty(ctx.n)
    out = ctx.empty(3)
    ctx.call("psc_lda_xc", _p(rho), _p(vxc), ctx.h ** 3, _p(out), _stream())
    return vxc, out


class Mixer:
    """msecant1 mixer with its history in device memory (Mixer/msecant1.py)."""

    def __init__(self, ctx: GridContext, capacity: int, mix: float = 0.5, restart_factor: float = 0.1):
        self.ctx, self.mix, self.rf = ctx, mix, restart_factor
        ctx.call("psc_mixer_reset", int(capacity))

    def __call__(self, x1: torch.Tensor, f1: torch.Tensor):
        out = torch.empty_like(x1)
        m = c_int()
        self.ctx.call("psc_mixer_step", _p(x1), _p(f1), self.mix, self.rf, _p(out), byref(m), _stream())
        return out, m.value


def qinv_from_gram(G: np.ndarray, tol: float) -> np.ndarray:
    """C = qinv(A) qinv(A)^T of Mixer/qinv.py:5-62 from G = A^T A (r x r) and
    tol = eps ||A||_inf.  qinv pivots A's columns by their remaining norms
    and cuts the rank at the first |R_ii| < tol; the pivoted Cholesky of G
    makes the same choices (its remaining diagonal is the squared remaining
    column norm, ties to the first column as LAPACK's) and gives the same
    |R_ii|.  C = P (S S^T) P^T with S = R11^{-1}, whatever the signs of R's
    rows.  The Gram matrix resolves a column's remaining norm only down to
    about sqrt(eps) of that column's own norm; a column whose remaining norm
    is below 8 sqrt(eps) of its norm is rounding noise of a dependent column
    and is cut there as well (the QR resolves down to tol itself; between
    the two the reference's coefficients are 1 / |R_ii|^2 amplifications of
    its own rounding).  Columns that are merely small are kept: late in an
    SCF the newest residual differences are many decades below the first."""
    G = 0.5 * (G + G.T)
    r = G.shape[0]
    norm0 = np.sqrt(np.maximum(np.diag(G), 0.0))
    floor = 8.0 * np.sqrt(np.finfo(float).eps)
    piv = np.arange(r)
    R = np.zeros((r, r))
    rank = r
    for j in range(r):
        p = j + int(np.argmax(np.diag(G)[j:]))
        if p != j:
            G[[j, p], :] = G[[p, j], :]
            G[:, [j, p]] = G[:, [p, j]]
            R[:j, [j, p]] = R[:j, [p, j]]
            piv[[j, p]] = piv[[p, j]]
        d = np.sqrt(max(G[j, j], 0.0))
        if d < tol or d <= floor * norm0[piv[j]]:
            rank = j
            break
        R[j, j] = d
        R[j, j + 1:] = G[j, j + 1:] / d
        G[j + 1:, j + 1:] -= np.outer(R[j, j + 1:], R[j, j + 1:])
    C = np.zeros((r, r))
    if rank:
        S = np.linalg.solve(R[:rank, :rank], np.eye(rank))   # R11 upper triangular: back substitution
        C[np.ix_(piv[:rank], piv[:rank])] = S @ S.T
    return C


class Mixer2:
    """Type-II multisecant mixer, Mixer/msecant2.py:24-93 with the parameters
    of Mixer/includemix.py:21-49; group_size 0 takes all iterates as one
    group (Anderson mixing).  The history (one FP64 n-vector pair per
    iterate) stays in device memory and every n-vector operation is a libpsc
    kernel (psc_mix2_*, psc_block_*, psc_gram, psc_gemm_nn); the host follows
    the reference's control flow: the restart test, the EN stages (a restart
    sets stage 2, after which the stages alternate, msecant2.py:45-93), the
    groups, and the quasi-inverse of the last group from its Gram matrix
    (qinv_from_gram)."""

    def __init__(self, ctx: GridContext, capacity: int, mix: float = 0.5, group_size: int = 0,
                 restart_factor: float = 0.1, en_like: int = 0):
        self.ctx, self.mix, self.gs, self.rf, self.en_like = ctx, mix, int(group_size), restart_factor, en_like
        self.cap = int(capacity) + 1
        self.DX = ctx.empty(self.cap, ctx.n)
        self.DF = ctx.empty(self.cap, ctx.n)
        self.coef = ctx.empty(self.cap)
        self.scal = ctx.empty(4)
        self.m = 0
        self.en = None

    def _dots(self, A: torch.Tensor, i0: int, r: int, x: torch.Tensor) -> torch.Tensor:
        self.ctx.call("psc_block_dots", _p(A[i0]), self.ctx.n, r, _p(x), _p(self.coef), _stream())
        return self.coef[:r]

    def _combine(self, y, base, f, mix, A=None, i0=0, r=0, c=None):
        self.ctx.call("psc_block_combine", _p(y), _p(base), _p(f), float(mix), _p(A[i0]) if r else None,
                      self.ctx.n, r, _p(c) if r else None, _stream())

    def __call__(self, x1: torch.Tensor, f1: torch.Tensor):
        ctx, mix, n = self.ctx, self.mix, self.ctx.n
        out = torch.empty_like(x1)
        if self.m == 0:
            ctx.call("psc_mix2_store", _p(x1), _p(f1), _p(self.DX[0]), _p(self.DF[0]), _stream())
            self._combine(out, x1, f1, mix)
            self.m, self.en = 1, (0 if self.en_like == 0 else 2)
            return out, 0
        m = self.m
        sz = m + 1 if self.gs == 0 else self.gs
        if self.en != 1 and m >= 2:
            ctx.call("psc_dot", _p(self.DF[m - 1]), _p(self.DF[m - 1]), n, _p(self.scal[0:1]), _stream())
            ctx.call("psc_dot", _p(f1), _p(f1), n, _p(self.scal[1:2]), _stream())
            nd, nf = np.sqrt(self.scal[:2].cpu().numpy())
            if nd < self.rf * nf:
                ctx.call("psc_mix2_store", _p(x1), _p(f1), _p(self.DX[0]), _p(self.DF[0]), _stream())
                self._combine(out, x1, f1, mix)
                self.m, self.en = 1, 2
                return out, 0
        if m + 1 > self.cap:
            raise PscError("mixer: history capacity exceeded")
        res = (m + sz - 1) % sz + 1
        ngroup = (m - res) // sz
        g = ngroup * sz
        if self.en != 1:
            ctx.call("psc_mix2_diff", _p(x1), _p(f1), _p(self.DX[m - 1]), _p(self.DF[m - 1]), float(mix),
                     _stream())
            if g:
                c = self._dots(self.DF, 0, g, self.DF[m - 1])
                self._combine(self.DX[m - 1], self.DX[m - 1], None, 0.0, self.DX, 0, g, c)
        if g:
            c = self._dots(self.DF, 0, g, f1)
            self._combine(out, x1, f1, mix, self.DX, 0, g, c)
        else:
            self._combine(out, x1, f1, mix)
        if self.en == 1 and res == sz:
            c = self._dots(self.DF, g, m - g, f1)
            self._combine(out, out, None, 0.0, self.DX, g, m - g, c)
        else:
            i0 = m - res
            G = ctx.empty(res, res)
            ctx.call("psc_gram", F64, _p(self.DF[i0]), n, _p(self.DF[i0]), n, res, 0, _p(G), _stream())
            ctx.call("psc_block_absrow_max", _p(self.DF[i0]), n, res, _p(self.scal[2:3]), _stream())
            Gh = G.cpu().numpy().reshape(res, res).T.copy()
            tol = np.finfo(float).eps * float(self.scal[2].item())
            C = qinv_from_gram(Gh, tol)
            if res == sz:
                Cd = torch.from_numpy(np.asfortranarray(C).ravel(order="F").copy()).to(ctx.device)
                tmp = torch.empty(res, n, dtype=torch.float64, device=ctx.device)
                ctx.call("psc_gemm_nn", F64, _p(self.DF[i0]), n, res, _p(Cd), res, _p(tmp), n, _stream())
                self.DF[i0:m].copy_(tmp)
                c = self._dots(self.DF, i0, res, f1)
            else:
                d = self._dots(self.DF, i0, res, f1).cpu().numpy()
                c = torch.from_numpy(C @ d).to(ctx.device)
            self._combine(out, out, None, 0.0, self.DX, i0, res, c)
        if self.en != 2:
            ctx.call("psc_mix2_store", _p(x1), _p(f1), _p(self.DX[m]), _p(self.DF[m]), _stream())
            self.m = m + 1
        if self.en == 1:
            self.en = 2
        elif self.en == 2:
            self.en = 1
        return out, m


def sad_setup(ctx: GridContext, atoms, elem, tables, ml_grid: bool = False):
    """SAD density, local and SAD Hartree potentials (V_ion/pseudoDiag.py).
    ml_grid: grid point i at i h instead of i h - radius, as
    V_ion/pseudoDiag_MLgrid.py (the same arithmetic with the radius 0)."""
    sp, xyz = ctx.atom_arrays(atoms, elem, tables)
    z_sum = 0.0
    for a in atoms:
        z_sum += elem[a["typ"]]["Z"] * np.asarray(a["coord"]).reshape(-1, 3).shape[0]
    rho0, hpot0, ppot = ctx.empty(ctx.n), ctx.empty(ctx.n), ctx.empty(ctx.n)
    info = (ctypes.c_double * 2)()
    h = ctx.h
    ctx.call("psc_sad_setup", len(sp), sp.ctypes.data_as(c_void_p), xyz.ctypes.data_as(c_void_p),
             0.0 if ml_grid else ctx.radius,
             h ** 3, 4 * np.pi, float(z_sum), _p(rho0), _p(hpot0), _p(ppot), info, _stream())
    diag_info = {"electron_count_initial": info[0], "electron_count_normalized": info[1],
                 "electron_target": float(z_sum)}
    return rho0, hpot0, ppot, diag_info


def projector_setup(ctx: GridContext, atoms, elem, tables, ml_grid: bool = False) -> NonlocalProjectors:
    """KB projectors (V_ion/pseudoNL_original.py); ml_grid as
    pseudoNL_original_MLgrid.py / pseudoNL_original_ML4Den.py (radius 0)."""
    sp, xyz = ctx.atom_arrays(atoms, elem, tables)
    ctx.call("psc_projector_setup", len(sp), sp.ctypes.data_as(c_void_p), xyz.ctypes.data_as(c_void_p),
             0.0 if ml_grid else ctx.radius, _stream())
    ctx.projectors = NonlocalProjectors(ctx)
    return ctx.projectors


def ml_density_setup(ctx: GridContext, atoms, elem, tables, density_file: str, cg_prec: int = 0):
    """The density-file start, V_ion/pseudoDiag_ML4Den_poisson.py:12-586:
    SAD on the ML grid, the file's density (1/A^3, shape (nx, ny, nz), read
    in Fortran order) converted to electrons per point, clamped at zero and
    renormalised, and its Hartree potential by CG from zero (preconditioned
    when cg_prec): returns (rho1, hpot0 + dV_H, ppot, diag_info)."""
    rho0, hpot0, ppot, _ = sad_setup(ctx, atoms, elem, tables, ml_grid=True)
    arr = np.load(density_file)
    if arr.ndim != 3 or arr.shape != (ctx.nx, ctx.ny, ctx.nz):
        raise ValueError(f"density file shape {arr.shape} does not match the grid {(ctx.nx, ctx.ny, ctx.nz)}")
    raw = torch.from_numpy(np.ascontiguousarray(np.ravel(np.asarray(arr, dtype=np.float64), order="F"))).to(ctx.device)
    z_sum = 0.0
    for a in atoms:
        z_sum += elem[a["typ"]]["Z"] * np.asarray(a["coord"]).reshape(-1, 3).shape[0]
    h = ctx.h
    a0 = 0.529177210903
    rho1, hrhs = ctx.empty(ctx.n), ctx.empty(ctx.n)
    info = (ctypes.c_double * 3)()
    ctx.call("psc_ml_density", _p(raw), a0 ** 3, h ** 3, float(z_sum), _p(rho0), 4 * np.pi / h ** 3, _p(rho1),
             _p(hrhs), info, _stream())
    prec = ("spectral", "precLU") if cg_prec else ()
    dh, _ = pcg(Laplacian(ctx), hrhs, ctx.zeros(ctx.n), 200, 1e-5, *prec)
    hpot1 = axpby(ctx, dh, hpot0, 1.0, 1.0)
    diag_info = {"electron_count_initial": info[0], "electron_count_normalized": info[2],
                 "electron_target": float(z_sum), "negative_values_zeroed": int(info[1])}
    return rho1, hpot1, ppot, diag_info


def scf_update(ctx, ppot, vxc, hpot, hpot0, rho, pot):
    """pot_new, f = pot_new - pot and [|f|^2, |pot_new|^2, sum rho(hpot+hpot0), sum rho vxc]."""
    pot_new, f, sums = ctx.empty(ctx.n), ctx.empty(ctx.n), ctx.empty(4)
    ctx.call("psc_scf_update", _p(ppot), _p(vxc), _p(hpot), _p(hpot0), _p(rho), _p(pot), _p(pot_new), _p(f),
             _p(sums), _stream())
    return pot_new, f, sums


def axpby(ctx, x, y, a, b):
    out = ctx.empty(ctx.n)
    ctx.call("psc_axpby", _p(x), _p(y), float(a), float(b), _p(out), ctx.n, _stream())
    return out


def numpy_sum(ctx, x) -> torch.Tensor:
    out = ctx.empty(1)
    ctx.call("psc_numpy_sum", _p(x), x.numel(), _p(out), _stream())
    return out


def nuclear(atoms, elem) -> float:
    """E_nuc = 2 sum_{i<j} Z_i Z_j / R_ij in Ry (Laplacian/nuclear.py:26-91)."""
    pts, zs = [], []
    for a in atoms:
        for row in np.asarray(a["coord"], dtype=float).reshape(-1, 3):
            pts.append(row)
            zs.append(elem[a["typ"]]["Z"])
    e = 0
    for i in range(len(pts)):
        for j in range(i + 1, len(pts)):
            d2 = (pts[i][0] - pts[j][0]) ** 2 + (pts[i][1] - pts[j][1]) ** 2 + (pts[i][2] - pts[j][2]) ** 2
            e += zs[i] * zs[j] / math.sqrt(d2)
    return float(e * 2)


def nelectrons(atoms, elem) -> int:
    return int(sum(elem[a["typ"]]["Z"] * np.asarray(a["coord"]).reshape(-1, 3).shape[0] for a in atoms))
