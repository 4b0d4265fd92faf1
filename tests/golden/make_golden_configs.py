"""Reference SCF results at the benchmark configurations (golden fixtures).

Runs PARSEC.py's own CPU SCF (rsdft_solver.run_rsdft_calculation) on the
synthetic geometry of one configuration (parsec_python_b200.workloads) with
numpy's global seed 0, and writes tests/golden/ref_<name>.npz: the final
energy components, eigenvalues, occupations, per-iteration total energies
and the converged density (float32, electrons per bohr^3).

Usage: python tests/golden/make_golden_configs.py NAME [reference src dir] [--tol T]
With --tol the fixture is written as ref_<name>_tol<exponent>.npz/.json.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
import time
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))


def main(name: str, src: str, tol: float | None = None) -> None:
    from parsec_python_b200 import workloads as w

    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)
    sys.path.insert(0, src)
    os.chdir(tempfile.mkdtemp())
    import rsdft_input
    import rsdft_solver
    from rsdft_backend import select_solver_backend
    from rsdft_models import A0_ANG, InputData, PreparedSystem, RunPaths, SolverSettings

    cfg = w.CONFIGS[name]
    atoms_ang = cfg["atoms"]()
    f = 1.0 / A0_ANG
    atoms = [{"typ": a["typ"], "coord": np.asarray(a["coord"], dtype=float) * f} for a in atoms_ang]
    h = cfg["h"] * f
    radius = cfg["radius"] * f
    nx = int(2 * radius / h) + 1
    nx = 2 * ((nx + 1) // 2)
    dom = {"radius": 0.5 * h * (nx - 1), "nx": nx, "ny": nx, "nz": nx, "h": h}
    elem, n_el = rsdft_input.load_elements(Path(src))
    tol = cfg["tol"] if tol is None else tol
    tag = name if tol == cfg["tol"] else f"{name}_tol{int(round(-np.log10(tol)))}"
    settings = SolverSettings(tol=tol, maxits=80, poldeg=cfg["poldeg"], fd_order=8)
    settings.normalize()
    tmp = Path(tempfile.mkdtemp())
    paths = RunPaths(output_file=str(tmp / "run.out"), wfn_file=str(tmp / "wfn.dat"),
                     initial_density_base=str(tmp / "init"), converged_density_base=str(tmp / "conv"))
    zel = float(sum(int(elem[elem["Element"] == a["typ"]]["Z"].iloc[0]) * len(a["coord"]) for a in atoms))
    inp = InputData(atoms=atoms, n_atom=[len(a["coord"]) for a in atoms], z_charge=0.0)
    prob = PreparedSystem(input_data=inp, settings=settings, domain=dom, h=h, nev=cfg["nev"], zelec=zel,
                          ztest=zel, n_types=len(atoms), paths=paths)
    np.random.seed(0)
    t0 = time.time()
    res = rsdft_solver.run_rsdft_calculation(prob, elem, n_el, select_solver_backend(settings))
    wall = time.time() - t0
    text = (tmp / "run.out").read_text()
    hist = [float(l.split("=")[2].split()[0]) for l in text.splitlines() if "Total electronic energy" in l]
    errs = [float(l.split("=")[1]) for l in text.splitlines() if "SCF error =" in l]
    fin = rsdft_solver.compute_energy_components(res.rho, res.hpot, res.hpot0, res.xc_potential, res.exc,
                                                 res.eigenvalues, res.occupations, cfg["nev"], res.e_nuc0, h)
    np.savez_compressed(HERE / f"ref_{tag}.npz", rho=res.rho.astype(np.float32), eigenvalues=res.eigenvalues,
                        occupations=res.occupations, total_ry=np.array(fin.total_ry),
                        eigen_sum_ry=np.array(fin.eigen_sum_ry), hartree_ry=np.array(fin.hartree_ry),
                        xc_ry=np.array(fin.xc_ry), ion_ry=np.array(fin.ion_ry), log_total_ry=np.array(hist[:-1]),
                        log_err=np.array(errs))
    meta = {"name": name, "domain": dom, "nev": cfg["nev"], "poldeg": cfg["poldeg"], "tol": tol, "seed": 0,
            "iterations": res.iterations, "error": float(res.error), "converged": bool(res.converged),
            "wall_s": wall, "total_ry": fin.total_ry, "cpu": os.cpu_count()}
    (HERE / f"ref_{tag}.json").write_text(json.dumps(meta, indent=1))
    print(json.dumps(meta))


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--tol")]
    tols = [float(a.split("=", 1)[1]) for a in sys.argv[1:] if a.startswith("--tol=")]
    src = args[1] if len(args) > 1 else os.environ.get("PARSEC_REF_SRC")
    if not args or not src:
        sys.exit(f"usage: python {sys.argv[0]} NAME <reference src directory> [--tol=T] (or set PARSEC_REF_SRC)")
    main(args[0], src, tols[0] if tols else None)
