"""B200-native real-space Kohn-Sham SCF hot path (PARSEC.py's use_gpu=1 path).

The compute path is libpsc.so (hand-written sm_100a CUDA kernels behind the
C ABI in include/psc.h); this package is the Python host side mirroring the
reference's backend bundle, SCF driver and input/output formats.
"""
from .models import (A0_ANG, RY_EV, EnergyComponents, InputData, PreparedSystem, RunPaths, SCFResult,  # noqa: F401
                     SolverBackend, SolverSettings)

__all__ = ["SolverSettings", "InputData", "PreparedSystem", "RunPaths", "SolverBackend", "EnergyComponents",
           "SCFResult", "select_solver_backend", "run_rsdft_calculation", "A0_ANG", "RY_EV"]


def select_solver_backend(settings):
    from .backend import select_solver_backend as _sel
    return _sel(settings)


def run_rsdft_calculation(problem, elem, n_elements, backend, **kw):
    from .solver import run_rsdft_calculation as _run
    return _run(problem, elem, n_elements, backend, **kw)
