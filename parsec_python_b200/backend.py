"""Backend selection: the GPU bundle behind the reference's entry points.

``select_solver_backend(settings)`` returns a ``SolverBackend`` with the
callables PARSEC.py's rsdft_backend.select_solver_backend
(rsdft_backend.py:80-137) provides for ``use_gpu = 1`` -- pseudo_diag,
pseudo_nl, first_filt, chefsi1, lanczos, chsubsp, occupations, pcg -- with
the same argument meaning.  They run on libpsc.so; there is no CPU path, and
as in the reference a GPU that cannot be used ends the run with SystemExit.
"""
from __future__ import annotations

import torch

from . import gpu
from .inputs import pseudo_tables
from .models import SolverBackend, SolverSettings


class GpuRuntime:
    """Per-run device state: one grid context per domain, precision, seeds."""

    def __init__(self, settings: SolverSettings):
        self.settings = settings
        self.block_dtype = torch.float32 if settings.precision == "mixed" else torch.float64
        self.ctx: gpu.GridContext | None = None

    def context(self, domain: dict) -> gpu.GridContext:
        if self.ctx is None or not self.ctx.matches(domain, self.settings.fd_order):
            self.ctx = gpu.GridContext(domain, self.settings.fd_order, seed=self.settings.seed)
            if self.settings.mask == "sphere":
                # the sphere inscribed in the cube: radius = the domain's half-width
                self.ctx.set_sphere_mask(self.ctx.radius)
        return self.ctx

    # -- reference entry points ------------------------------------------------
    def pseudo_diag(self, domain, atoms, elem, n_elements=None, return_info=False):
        ctx = self.context(domain)
        rho0, hpot0, ppot, info = gpu.sad_setup(ctx, atoms, elem, pseudo_tables())
        return (rho0, hpot0, ppot, info) if return_info else (rho0, hpot0, ppot)

    def pseudo_nl(self, domain, atoms, elem, n_elements=None):
        return gpu.projector_setup(self.context(domain), atoms, elem, pseudo_tables())

    # the ML-grid setups, imported directly by the reference's driver
    # (rsdft_solver.py:89-108,118-127)
    def pseudo_diag_mlgrid(self, domain, atoms, elem, n_elements=None, return_info=False):
        ctx = self.context(domain)
        rho0, hpot0, ppot, info = gpu.sad_setup(ctx, atoms, elem, pseudo_tables(), ml_grid=True)
        return (rho0, hpot0, ppot, info) if return_info else (rho0, hpot0, ppot)

    def pseudo_nl_mlgrid(self, domain, atoms, elem, n_elements=None):
        return gpu.projector_setup(self.context(domain), atoms, elem, pseudo_tables(), ml_grid=True)

    def pseudo_diag_ml4den(self, domain, atoms, elem, n_elements, density_file, A=None, cg_prec=0, PRE=None,
                           return_info=False):
        ctx = self.context(domain)
        rho1, hpot1, ppot, info = gpu.ml_density_setup(ctx, atoms, elem, pseudo_tables(), density_file, cg_prec)
        return (rho1, hpot1, ppot, info) if return_info else (rho1, hpot1, ppot)

    def first_filt(self, nev, H, polm=10):
        s = self.settings
        return gpu.first_filt(nev, H, polm, dtype=self.block_dtype, energ_tol=s.first_tol,
                              max_iter=s.first_rounds or None)

    def chefsi1(self, W, ritzv, deg, nev, H):
        return gpu.chefsi1(W, ritzv, deg, nev, H)

    def lanczos(self, B, nev, v, m, tol, *args):
        """Eigensolvers/lanczos.py:10 signature; v None draws the start on the device."""
        return gpu.lanczos(B, nev, v, m, tol, dtype=self.block_dtype)

    def chsubsp(self, deg, nev, H):
        return gpu.chsubsp(deg, nev, H, dtype=self.block_dtype)

    def occupations(self, lam, temp, nelec, tol):
        return gpu.occupations(self.ctx, lam, temp, nelec, tol)

    def pcg(self, A, rhs, x0, maxit, tol, *prec):
        return gpu.pcg(A, rhs, x0, maxit, tol, *prec)


def select_solver_backend(settings: SolverSettings) -> SolverBackend:
    if not settings.use_gpu:
        raise SystemExit("this implementation has only the GPU backend (use_gpu = 1)")
    try:
        gpu.require_cuda()
    except Exception as exc:  # same contract as the reference: no usable GPU -> SystemExit
        raise SystemExit(f"GPU backend requested but unavailable: {exc}") from exc
    rt = GpuRuntime(settings)
    return SolverBackend(label="gpu", pseudo_diag=rt.pseudo_diag, pseudo_nl=rt.pseudo_nl, first_filt=rt.first_filt,
                         chefsi1=rt.chefsi1, lanczos=rt.lanczos, chsubsp=rt.chsubsp, occupations=rt.occupations,
                         pcg=rt.pcg, array_module=torch, cupy_module=None, runtime=rt)
