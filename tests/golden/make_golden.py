"""Generate the golden fixtures that pin the oracle to the reference.

Runs PARSEC.py's own CPU code (zeyizhang-berkeley/parsec_python, ``src/``)
in this container -- it needs only numpy, scipy and pandas plus a stub for the
unused ``matplotlib`` import -- on small seeded inputs, and writes the outputs
to ``tests/golden/ref_*.npz`` and ``tests/golden/ref_meta.json``.  Machines
that run the tests need no copy of the reference: the tests read only these
files.

Usage: python tests/golden/make_golden.py [reference src dir]
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile
import time
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
A0 = 0.529177210903


def _import_reference(src: str):
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)
    sys.path.insert(0, src)


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def h2o_atoms(angstrom_coords):
    o = np.array([angstrom_coords[0]], dtype=float) / A0
    hh = np.array(angstrom_coords[1:], dtype=float) / A0
    return [{"typ": "O", "coord": o}, {"typ": "H", "coord": hh}]


def small_domain(h, radius):
    nx = int(2 * radius / h) + 1
    nx = 2 * ((nx + 1) // 2)
    return {"radius": 0.5 * h * (nx - 1), "nx": nx, "ny": nx, "nz": nx, "h": h}


def main(src: str) -> None:
    _import_reference(src)
    os.chdir(tempfile.mkdtemp())  # pseudoDiag appends to ./error_log.txt
    from Laplacian.fd3d import fd3d
    from V_ion.pseudoDiag import pseudoDiag
    from V_ion.pseudoNL_original import pseudoNL
    from V_ion.splineData import splineData
    from V_ion.preProcess import preProcess
    from Splines.fspline import fspline
    from Splines.fsplevalIO import fsplevalIO
    from V_xc.exc_nspn import exc_nspn
    from Mixer import msecant1 as ms1
    from Eigensolvers.occupations import occupations
    from Eigensolvers.pcg import pcg
    from Eigensolvers.lancz_uppbnd import lancz_uppbnd
    from Eigensolvers.lanczosForChefsi1 import lanczosForChefsi1
    from Eigensolvers.first_filt import first_filt
    from Eigensolvers.chefsi1 import chefsi1
    from Laplacian.nuclear import nuclear
    import rsdft_input
    import rsdft_solver
    from rsdft_models import InputData, PreparedSystem, RunPaths, SolverSettings
    from rsdft_backend import select_solver_backend

    elem, n_el = rsdft_input.load_elements(Path(src))
    meta: dict = {"elements": {}}
    for i in range(n_el):
        meta["elements"][elem["Element"].iloc[i]] = [float(elem[c].iloc[i]) for c in
                                                     ("Z", "Zvalue", "h", "r", "R")]
    rng = np.random.default_rng(1234)

    # ---- finite-difference Laplacian (Laplacian/fd3d.py) ----
    fd = {}
    for (nx, ny, nz, order) in [(7, 6, 5, 8), (6, 6, 6, 6), (5, 7, 6, 4), (6, 5, 7, 2), (2, 2, 2, 8),
                                (3, 4, 5, 8), (9, 9, 9, 8)]:
        n = nx * ny * nz
        x = rng.standard_normal((n, 3))
        y = fd3d(nx, ny, nz, order) @ x
        key = f"{nx}_{ny}_{nz}_{order}"
        fd[f"x_{key}"] = x
        fd[f"y_{key}"] = y
    np.savez_compressed(HERE / "ref_fd3d.npz", **fd)

    # ---- splines (Splines/*, V_ion/preProcess.py) ----
    tables, labels = splineData()
    spl = {}
    meta["splines"] = {}
    for entry in tables:
        el = entry["atom"]
        if el not in ("H", "C", "O", "Si"):
            continue
        data = entry["data"]
        cols = {"charge": data[:, 1], "hartree": data[:, 2], "pot_S": data[:, 4],
                "wfn_P": data[:, 5], "potPS": data[:, 3] - data[:, 4]}
        for name, y in cols.items():
            I = preProcess(y)
            xk, yk = data[:, 0][I], y[I]
            z, c, d = fspline(xk, yk)
            r = np.concatenate([[0.0, 1e-7], np.linspace(0.0, 12.0, 397), [200.0]])
            vals = np.empty_like(r)
            j = 0
            for t, rv in enumerate(r):
                vals[t], j = fsplevalIO(z, c, d, xk, rv, j)
            tag = f"{el}_{name}"
            spl[f"r_{tag}"] = r
            spl[f"v_{tag}"] = vals
            meta["splines"][tag] = {"keep": sha(np.asarray(I, dtype=np.int64)), "z": sha(z), "c": sha(c),
                                    "d": sha(d), "nknots": int(len(I))}
    np.savez_compressed(HERE / "ref_splines.npz", **spl)

    # ---- ionic setup on a small H2O box (V_ion/pseudoDiag.py, pseudoNL_original.py) ----
    atoms = h2o_atoms([(0.0, 0.0, 0.0), (0.757, 0.586, 0.0), (-0.757, 0.586, 0.0)])
    dom = small_domain(0.45, 5.0)
    rho0, hpot0, ppot, info = pseudoDiag(dom, atoms, elem, n_el, return_info=True)
    vnl = pseudoNL(dom, atoms, elem, n_el).tocsr()
    n = dom["nx"] ** 3
    xn = rng.standard_normal((n, 2))
    ion = {"rho0": rho0, "hpot0": hpot0, "ppot": ppot, "vnl_x": xn, "vnl_y": vnl @ xn}
    np.savez_compressed(HERE / "ref_ion_h2o.npz", **ion)
    meta["ion_h2o"] = {"domain": dom, "atoms": [[a["typ"], a["coord"].tolist()] for a in atoms],
                       "rho0": sha(rho0), "hpot0": sha(hpot0), "ppot": sha(ppot), "info": info,
                       "e_nuc": float(nuclear(dom, atoms, elem, n_el))}

    # ---- shipped H2O sample: SAD density known-answer test ----
    sample = Path(src).parent / "samples" / "h2o"
    init_grid = np.load(sample / "H2O_sad_diagmeth3_5A_0p2A_init_rho_grid.npy")
    meta["sample_h2o_init_rho_grid"] = {"sha256": sha(init_grid), "shape": list(init_grid.shape),
                                        "sum": float(init_grid.sum())}

    # ---- LDA XC (V_xc/exc_nspn.py) ----
    rho = np.concatenate([np.zeros(5), -np.abs(rng.standard_normal(5)) * 1e-3,
                          10 ** rng.uniform(-9, 1.5, 1990)])
    vxc, exc = exc_nspn({"h": 0.37}, rho.copy())
    np.savez_compressed(HERE / "ref_xc.npz", rho=rho, vxc=vxc, exc=np.array(exc))

    # ---- msecant1 mixer (Mixer/msecant1.py) ----
    mx = ms1.mixer()
    nmix = 64
    amat = rng.standard_normal((nmix, nmix)) * 0.2 / np.sqrt(nmix)
    bvec = rng.standard_normal(nmix)
    x = rng.standard_normal(nmix)
    xs, fs, outs = [], [], []
    for step in range(14):
        f = np.tanh(amat @ x) + bvec - x
        if step == 9:
            f = f * 50.0     # forces the restart branch (|df_last| < 0.1 |f|)
        xs.append(x.copy())
        fs.append(f.copy())
        x, _ = mx.mixer(x, f)
        outs.append(np.asarray(x).copy())
    np.savez_compressed(HERE / "ref_mixer.npz", x=np.array(xs), f=np.array(fs), out=np.array(outs))

    # ---- occupations (Eigensolvers/occupations.py) ----
    occ_cases = {}
    lam_sets = [np.sort(rng.uniform(-1.0, 0.5, 12)), np.linspace(-0.9, -0.1, 12),
                np.array([-0.5, -0.4, -0.3, -0.3, -0.29, -0.2, 0.1, 0.2]),
                np.array([-1.0, -0.8, -0.7])]
    nelecs = [8, 8, 7, 20]
    for i, (lam, ne) in enumerate(zip(lam_sets, nelecs)):
        c, occv = occupations(lam.copy(), 500.0, ne, 1e-6)
        occ_cases[f"lam_{i}"] = lam
        occ_cases[f"ne_{i}"] = np.array(ne)
        occ_cases[f"ef_{i}"] = np.array(c)
        occ_cases[f"occ_{i}"] = np.asarray(occv)
    np.savez_compressed(HERE / "ref_occupations.npz", **occ_cases)

    # ---- Hartree CG (Eigensolvers/pcg.py) ----
    A = (1.0 / (0.4 * 0.4)) * fd3d(10, 10, 10, 8)
    rhs = rng.standard_normal(1000)
    x0 = rng.standard_normal(1000) * 0.1
    xs_, its = pcg(A, rhs, x0, 200, 1e-5)
    np.savez_compressed(HERE / "ref_pcg.npz", rhs=rhs, x0=x0, x=xs_, its=np.array(its))

    # ---- Lanczos bounds and the two filter drivers on the small H2O Hamiltonian ----
    import scipy.sparse as sp
    Afull = (1.0 / (dom["h"] ** 2)) * fd3d(dom["nx"], dom["ny"], dom["nz"], 8)
    pot = ppot + hpot0
    B = (0.5 * Afull + vnl + sp.diags(pot, 0, shape=(n, n))).tocsr()
    np.random.seed(7)
    ub, ritz = lancz_uppbnd(n, B)
    np.random.seed(8)
    bound = lanczosForChefsi1(B, 6, np.random.randn(n, 1), 6, 0.0)
    np.random.seed(9)
    W, lam = first_filt(27, B, 10)
    np.random.seed(10)
    W2, lam2 = chefsi1(W, lam, 10, 12, B)
    np.savez_compressed(HERE / "ref_eigs.npz", uppbnd=np.array(ub), ritz=ritz, bound=np.array(bound),
                        ff_lam=lam, cf_lam=lam2, cf_rho=(W2[:, :12] ** 2).sum(axis=1), pot=pot)

    # ---- full SCF, small H2O (rsdft_solver.run_rsdft_calculation) ----
    settings = SolverSettings(tol=1e-6, maxits=40, poldeg=10, fd_order=8)
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
    out_text = (tmp / "h2o.out").read_text()
    energies = [float(line.split("=")[2].split()[0]) for line in out_text.splitlines()
                if "Total electronic energy" in line]
    from rsdft_solver import compute_energy_components
    fin = compute_energy_components(res.rho, res.hpot, res.hpot0, res.xc_potential, res.exc,
                                    res.eigenvalues, res.occupations, 12, res.e_nuc0, dom_scf["h"])
    np.savez_compressed(HERE / "ref_scf_h2o.npz", rho=res.rho, eigenvalues=res.eigenvalues,
                        occupations=res.occupations, total_ry=np.array(fin.total_ry),
                        eigen_sum_ry=np.array(fin.eigen_sum_ry), hartree_ry=np.array(fin.hartree_ry),
                        xc_ry=np.array(fin.xc_ry), log_total_ry=np.array(energies), hpot=res.hpot)
    meta["scf_h2o"] = {"domain": dom_scf, "nev": 12, "poldeg": 10, "tol": 1e-6, "seed": 0,
                       "iterations": res.iterations, "error": float(res.error), "wall_s": wall,
                       "total_ry": fin.total_ry}
    (HERE / "ref_meta.json").write_text(json.dumps(meta, indent=1, default=float))
    print("golden fixtures written; scf iterations", res.iterations, "E", fin.total_ry, "wall", wall)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("PARSEC_REF_SRC"):
        main(os.environ["PARSEC_REF_SRC"])
    else:
        sys.exit(f"usage: python {sys.argv[0]} <reference src directory> (or set PARSEC_REF_SRC)")
