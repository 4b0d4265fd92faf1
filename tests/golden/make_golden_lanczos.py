"""Generate the golden fixtures that pin the oracle's Lanczos-based
eigensolvers (diagmeth 0/1/2) to the reference.

Runs PARSEC.py's own CPU code (zeyizhang-berkeley/parsec_python, ``src/``):
``Eigensolvers/lanczosForChsubsp.py``, ``Eigensolvers/chsubsp.py`` and
``Eigensolvers/lanczos.py`` on the Hamiltonian of a small H2O box, seeded, and
a full SCF with diagmeth = 2, and writes ``tests/golden/ref_lanczos.npz`` and
``tests/golden/ref_lanczos.json``.  ``lanczos.py`` is run where it can run:
for n <= 35000 its convergence test assigns into an empty list and raises
IndexError, which is recorded in the JSON.

Usage: python tests/golden/make_golden_lanczos.py [reference src dir]
"""
from __future__ import annotations

import json
import os
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_golden import _import_reference, h2o_atoms, small_domain, sha  # noqa: E402

A0 = 0.529177210903


def hamiltonian(dom, atoms, elem, n_el):
    import scipy.sparse as sp
    from Laplacian.fd3d import fd3d
    from V_ion.pseudoDiag import pseudoDiag
    from V_ion.pseudoNL_original import pseudoNL

    rho0, hpot0, ppot = pseudoDiag(dom, atoms, elem, n_el)
    vnl = pseudoNL(dom, atoms, elem, n_el).tocsr()
    n = dom["nx"] * dom["ny"] * dom["nz"]
    A = (1.0 / (dom["h"] ** 2)) * fd3d(dom["nx"], dom["ny"], dom["nz"], 8)
    pot = ppot + hpot0
    return (0.5 * A + vnl + sp.diags(pot, 0, shape=(n, n))).tocsr(), pot


def main(src: str) -> None:
    _import_reference(src)
    os.chdir(tempfile.mkdtemp())
    from Eigensolvers.chsubsp import chsubsp
    from Eigensolvers.lanczos import lanczos
    from Eigensolvers.lanczosForChsubsp import lanczosForChsubsp
    import rsdft_input
    import rsdft_solver
    from rsdft_backend import select_solver_backend
    from rsdft_models import InputData, PreparedSystem, RunPaths, SolverSettings

    elem, n_el = rsdft_input.load_elements(Path(src))
    atoms = h2o_atoms([(0.0, 0.0, 0.0), (0.757, 0.586, 0.0), (-0.757, 0.586, 0.0)])
    out: dict = {}
    meta: dict = {}

    # ---- n <= 35000: lanczosForChsubsp with its convergence test, chsubsp ----
    dom = small_domain(0.45, 5.0)
    B, pot = hamiltonian(dom, atoms, elem, n_el)
    n = B.shape[0]
    out["small_pot"] = pot
    np.random.seed(21)
    v = np.random.randn(n)
    W, lam, bound = lanczosForChsubsp(B, 27, v.copy(), 450)
    out.update(small_v=v, small_lfc_lam=lam, small_lfc_bound=np.array(bound),
               small_lfc_rho4=(W[:, :4] ** 2).sum(axis=1))
    meta["small"] = {"domain": dom, "n": n, "nev": 27, "m": 450, "lfc_W": sha(W)}
    np.random.seed(22)
    W, ritz = chsubsp(10, 27, B)
    out.update(small_ch_ritz=ritz, small_ch_rho4=(W[:, :4] ** 2).sum(axis=1))
    meta["small"]["chsubsp_seed"] = 22
    np.random.seed(23)
    try:
        lanczos(B, 27, np.random.randn(n, 1), 12 + 500, 1e-5)
        meta["small"]["lanczos_cpu"] = "ran"
    except Exception as exc:  # the CPU lanczos cannot run its convergence test
        meta["small"]["lanczos_cpu"] = f"{type(exc).__name__}: {exc}"

    # ---- n > 35000: no convergence test in either routine ----
    dom = small_domain(0.3, 5.0)
    B, pot = hamiltonian(dom, atoms, elem, n_el)
    n = B.shape[0]
    assert n > 35000
    out["big_pot"] = pot
    np.random.seed(31)
    v = np.random.randn(n)
    W, lam, bound = lanczosForChsubsp(B, 27, v.copy(), 450)
    out.update(big_v=v, big_lfc_lam=lam, big_lfc_bound=np.array(bound), big_lfc_rho4=(W[:, :4] ** 2).sum(axis=1))
    np.random.seed(32)
    v = np.random.randn(n, 1)
    t0 = time.time()
    W, lam = lanczos(B, 27, v.copy(), 12 + 500, 1e-5)
    out.update(big_lz_v=v[:, 0], big_lz_lam=lam, big_lz_rho4=(W[:, :4] ** 2).sum(axis=1))
    meta["big"] = {"domain": dom, "n": n, "nev": 27, "m_lfc": 450, "m_lz": 512, "lfc_W": sha(W),
                   "lanczos_s": time.time() - t0}

    # ---- full SCF with diagmeth = 2 (chsubsp first, then chefsi1) ----
    settings = SolverSettings(tol=1e-6, maxits=40, poldeg=10, fd_order=8, diagmeth=2)
    settings.normalize()
    dom_scf = small_domain(0.3 / A0, 4.0 / A0)
    tmp = Path(tempfile.mkdtemp())
    inp = InputData(atoms=atoms, n_atom=[1, 2], z_charge=0.0)
    paths = RunPaths(output_file=str(tmp / "h2o.out"), wfn_file=str(tmp / "wfn.dat"),
                     initial_density_base=str(tmp / "init"), converged_density_base=str(tmp / "conv"))
    prob = PreparedSystem(input_data=inp, settings=settings, domain=dom_scf, h=dom_scf["h"], nev=12,
                          zelec=8.0, ztest=8.0, n_types=2, paths=paths)
    backend = select_solver_backend(settings)
    np.random.seed(0)
    t0 = time.time()
    res = rsdft_solver.run_rsdft_calculation(prob, elem, n_el, backend)
    wall = time.time() - t0
    from rsdft_solver import compute_energy_components
    fin = compute_energy_components(res.rho, res.hpot, res.hpot0, res.xc_potential, res.exc,
                                    res.eigenvalues, res.occupations, 12, res.e_nuc0, dom_scf["h"])
    out.update(scf2_eigenvalues=res.eigenvalues, scf2_total_ry=np.array(fin.total_ry), scf2_rho=res.rho)
    meta["scf_diagmeth2"] = {"domain": dom_scf, "nev": 12, "poldeg": 10, "tol": 1e-6, "seed": 0,
                             "iterations": res.iterations, "error": float(res.error), "wall_s": wall,
                             "total_ry": fin.total_ry}
    np.savez_compressed(HERE / "ref_lanczos.npz", **out)
    (HERE / "ref_lanczos.json").write_text(json.dumps(meta, indent=1, default=float))
    print(json.dumps(meta, indent=1, default=float))


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("PARSEC_REF_SRC"):
        main(os.environ["PARSEC_REF_SRC"])
    else:
        sys.exit(f"usage: python {sys.argv[0]} <reference src directory> (or set PARSEC_REF_SRC)")
