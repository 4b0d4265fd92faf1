"""H.X on the H2O configuration's grid from the reference's own operator.

Builds PARSEC.py's Hamiltonian B = 0.5 A + V_nl + diag(ppot + hpot0) with its
own fd3d, pseudoDiag and pseudoNL (the CSR matrix rsdft_solver.py:263,285
assembles) on the H2O configuration (O at the origin, H at (+-0.757, 0.586,
0) A, sphere radius 5 A, spacing 0.2 A: 52^3 = 140,608 points) and applies
it to two seeded standard-normal columns (numpy default_rng(11)).  Writes
tests/golden/ref_hx_h2o.npz: the potential and B X.

Usage: python tests/golden/make_golden_hx.py <reference src directory> (or set PARSEC_REF_SRC)
"""
from __future__ import annotations

import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))


def main(src: str) -> None:
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", plt)
    sys.path.insert(0, src)
    os.chdir(tempfile.mkdtemp())  # pseudoDiag appends to ./error_log.txt
    import scipy.sparse as sp
    import rsdft_input
    from Laplacian.fd3d import fd3d
    from V_ion.pseudoDiag import pseudoDiag
    from V_ion.pseudoNL_original import pseudoNL

    from parsec_python_b200 import workloads

    elem, n_el = rsdft_input.load_elements(Path(src))
    cfg = workloads.config_system("h2o")
    atoms, h, radius = cfg["atoms"], cfg["h"], cfg["radius"]
    nx = int(2 * radius / h) + 1  # rsdft_setup.py:133-150 with a radius override
    nx = 2 * ((nx + 1) // 2)
    dom = {"radius": 0.5 * h * (nx - 1), "nx": nx, "ny": nx, "nz": nx, "h": h}
    n = nx ** 3
    _, hpot0, ppot = pseudoDiag(dom, atoms, elem, n_el)
    vnl = pseudoNL(dom, atoms, elem, n_el).tocsr()
    pot = ppot + hpot0
    A = (1.0 / (h * h)) * fd3d(nx, nx, nx, 8)
    B = (0.5 * A + vnl + sp.diags(pot, 0, shape=(n, n))).tocsr()
    X = np.random.default_rng(11).standard_normal((n, 2))
    np.savez_compressed(HERE / "ref_hx_h2o.npz", pot=pot, y=B @ X, nx=np.array(nx), h=np.array(h),
                        radius=np.array(dom["radius"]))
    print(f"wrote ref_hx_h2o.npz: n = {n}, |B X| max = {np.abs(B @ X).max():.6g}")


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("PARSEC_REF_SRC"):
        main(os.environ["PARSEC_REF_SRC"])
    else:
        sys.exit(f"usage: python {sys.argv[0]} <reference src directory> (or set PARSEC_REF_SRC)")
