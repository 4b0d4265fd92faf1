"""Generate the fixtures that pin the oracle's ML-grid density modes
(density_method = sad_ml_grid and ml) to the reference.

Runs PARSEC.py's own CPU code (zeyizhang-berkeley/parsec_python, ``src/``) on
an H2O molecule in a 6 A POSCAR cell with a 24^3 grid: the ML-grid SAD setup
(V_ion/pseudoDiag_MLgrid.py), the ML-grid projectors
(V_ion/pseudoNL_original_MLgrid.py), the density-file start
(V_ion/pseudoDiag_ML4Den_poisson.py) and whole SCFs of both modes through the
reference's own input pipeline (rsdft_input.prepare_input_data,
rsdft_setup.prepare_system, rsdft_solver.run_rsdft_calculation).  The
density file is synthetic: the reference's own ML-grid SAD density in 1/A^3
with a smooth bump and a few negative values (which the reader clamps).
Writes tests/golden/ml/ (the input files) and tests/golden/ref_ml.npz /
ref_ml.json.

Usage: python tests/golden/make_golden_ml.py [reference src dir]
"""
from __future__ import annotations

import json
import os
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_golden import _import_reference, sha  # noqa: E402

A0 = 0.529177210903
L_ANG = 6.0
N = 24
# O and H (angstrom) inside the cell
ATOMS_ANG = [("O", [[3.0, 3.0, 3.1]]), ("H", [[3.757, 3.586, 3.1], [2.243, 3.586, 3.1]])]


def write_inputs(d: Path, density: np.ndarray, method: str) -> Path:
    d.mkdir(parents=True, exist_ok=True)
    (d / "cell.POSCAR").write_text(
        "H2O test cell\n1.0\n"
        f"{L_ANG:.6f} 0.000000 0.000000\n0.000000 {L_ANG:.6f} 0.000000\n0.000000 0.000000 {L_ANG:.6f}\n"
        "O H\n1 2\nCartesian\n3.0 3.0 3.1\n3.757 3.586 3.1\n2.243 3.586 3.1\n")
    np.save(d / "density.npy", density)
    lines = ["$system", "O 3.0 3.0 3.1", "H 3.757 3.586 3.1", "H 2.243 3.586 3.1", "$system", "$settings",
             "unit = Angstrom", f"density_method = {method}", "ml_file_path = density.npy",
             "grid_poscar_path = cell.POSCAR", "tol = 1e-6", "poldeg = 10", "nev = 12", "maxits = 60", "$settings"]
    inp = d / f"h2o_{method}.in"
    inp.write_text("\n".join(lines) + "\n")
    return inp


def main(src: str) -> None:
    _import_reference(src)
    os.chdir(tempfile.mkdtemp())
    from Laplacian.fd3d import fd3d
    from V_ion.pseudoDiag_MLgrid import pseudoDiag_MLgrid
    from V_ion.pseudoDiag_ML4Den_poisson import pseudoDiag_ML4Den
    from V_ion.pseudoNL_original_MLgrid import pseudoNL_MLgrid
    import rsdft_input
    import rsdft_setup
    import rsdft_solver
    from rsdft_backend import select_solver_backend
    from rsdft_models import SolverSettings

    elem, n_el = rsdft_input.load_elements(Path(src))
    h = L_ANG / N / A0
    dom = {"radius": L_ANG / 2 / A0, "nx": N, "ny": N, "nz": N, "h": h}
    atoms = [{"typ": t, "coord": np.array(c) / A0} for t, c in ATOMS_ANG]
    out: dict = {}
    meta: dict = {"domain": dom}

    rho0, hpot0, ppot, info = pseudoDiag_MLgrid(dom, atoms, elem, n_el, return_info=True)
    out.update(mlgrid_rho0=rho0, mlgrid_hpot0=hpot0, mlgrid_ppot=ppot)
    meta["mlgrid"] = {"rho0": sha(rho0), "hpot0": sha(hpot0), "ppot": sha(ppot), "info": info}
    vnl = pseudoNL_MLgrid(dom, atoms, elem, n_el).tocsr()
    x = np.random.default_rng(3).standard_normal((N ** 3, 2))
    out.update(vnl_x=x, vnl_y=vnl @ x)

    # synthetic density file: SAD density in 1/A^3, a smooth bump, a few negatives
    g = np.arange(N) * (L_ANG / N)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    sad = (rho0 / (L_ANG / N) ** 3).reshape(N, N, N, order="F")
    bump = 0.05 * np.exp(-((X - 3.4) ** 2 + (Y - 3.3) ** 2 + (Z - 3.0) ** 2) / 0.5)
    dens = sad + bump
    dens[0, 0, :4] = -1e-4
    out["density"] = dens

    A = (1.0 / h ** 2) * fd3d(N, N, N, 8)
    # the consumer reads the density from a file path
    tmp = Path(tempfile.mkdtemp())
    np.save(tmp / "d.npy", dens)
    rho1, hpot1, pot1, info1 = pseudoDiag_ML4Den(dom, atoms, elem, n_el, str(tmp / "d.npy"), A, return_info=True)
    out.update(ml_rho1=rho1, ml_hpot1=hpot1, ml_pot=pot1)
    meta["ml4den"] = {"info": info1, "rho1": sha(rho1), "pot": sha(pot1)}

    # whole SCFs through the reference's own input pipeline
    case_dir = HERE / "ml"
    for method in ("sad_ml_grid", "ml"):
        work = Path(tempfile.mkdtemp())
        inp = write_inputs(work, dens, method)
        settings = SolverSettings()
        settings.use_gpu = 0
        settings.normalize()
        data = rsdft_input.prepare_input_data(elem, settings, str(inp), base_dir=src)
        if not rsdft_input.has_diagmeth_override(data.settings_overrides):
            settings.diagmeth = 2
        settings.apply_overrides(data.settings_overrides)
        settings.use_gpu = 0
        settings.normalize()
        problem = rsdft_setup.prepare_system(data, settings, elem, n_el)
        backend = select_solver_backend(settings)
        np.random.seed(0)
        res = rsdft_solver.run_rsdft_calculation(problem, elem, n_el, backend)
        fin = rsdft_solver.compute_energy_components(res.rho, res.hpot, res.hpot0, res.xc_potential, res.exc,
                                                     res.eigenvalues, res.occupations, problem.nev, res.e_nuc0,
                                                     problem.domain["h"])
        out[f"scf_{method}_eigenvalues"] = res.eigenvalues
        out[f"scf_{method}_rho"] = res.rho
        meta[f"scf_{method}"] = {"domain": problem.domain, "nev": problem.nev, "diagmeth": settings.diagmeth,
                                 "iterations": res.iterations, "error": float(res.error), "total_ry": fin.total_ry}
        print(method, res.iterations, fin.total_ry)
        if method == "ml":
            # keep the input files the SCF read (small: POSCAR, .in, 24^3 density)
            if case_dir.exists():
                shutil.rmtree(case_dir)
            case_dir.mkdir()
            for f in ("cell.POSCAR", "density.npy", "h2o_ml.in"):
                shutil.copy(work / f, case_dir / f)
            (case_dir / "h2o_sad_ml_grid.in").write_text(
                (work / "h2o_ml.in").read_text().replace("density_method = ml", "density_method = sad_ml_grid"))
    np.savez_compressed(HERE / "ref_ml.npz", **out)
    (HERE / "ref_ml.json").write_text(json.dumps(meta, indent=1, default=float))
    print(json.dumps(meta, indent=1, default=float))


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("PARSEC_REF_SRC"):
        main(os.environ["PARSEC_REF_SRC"])
    else:
        sys.exit(f"usage: python {sys.argv[0]} <reference src directory> (or set PARSEC_REF_SRC)")
