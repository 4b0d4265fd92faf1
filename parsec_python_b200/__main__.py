"""Command line: python -m parsec_python_b200 INPUT [--precision fp64|mixed]

Runs one SCF on the GPU for an input file in the reference's formats and
writes the same .out log and density .npy files next to it
(PARSEC.py main_new.py:46-120).
"""
from __future__ import annotations

import argparse

from .backend import select_solver_backend
from .inputs import has_diagmeth_override, load_elements, prepare_input_data
from .models import SolverSettings
from .output import initialize_output_file, write_parameters
from .solver import run_rsdft_calculation
from .system import prepare_system


def main(argv=None):
    ap = argparse.ArgumentParser(description="B200 real-space Kohn-Sham SCF")
    ap.add_argument("input_file")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default=None)
    args = ap.parse_args(argv)
    settings = SolverSettings()
    settings.normalize()
    elem, n_el = load_elements()
    data = prepare_input_data(settings, args.input_file)
    if data.density_method in ("ml", "sad_ml_grid") and not has_diagmeth_override(data.settings_overrides):
        # main_new.py:76-78: ML density inputs default to chsubsp
        settings.diagmeth = 2
        print("No diagonalization override supplied for ML density input; using diagmeth=2 by default.")
    settings.apply_overrides(data.settings_overrides)
    if args.precision:
        settings.precision = args.precision
    settings.use_gpu = 1
    settings.normalize()
    backend = select_solver_backend(settings)
    problem = prepare_system(data, settings, elem, n_el)
    initialize_output_file(problem.paths.output_file, backend.label, problem.input_data.density_method)
    write_parameters(problem.paths.output_file, problem.nev, problem.input_data.atoms, problem.input_data.n_atom,
                     problem.domain, problem.h, settings.poldeg, settings.fd_order)
    return run_rsdft_calculation(problem, elem, n_el, backend)


if __name__ == "__main__":
    main()
