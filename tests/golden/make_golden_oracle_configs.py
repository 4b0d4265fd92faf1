"""Reference energies of the large benchmark configurations from the pinned oracle.

The reference's own CPU SCF takes many hours at Si87H76 (729,000 points,
292 states): its CSR products with the 38 M-entry projector blocks run
single-threaded.  This script runs the oracle instead -- the NumPy restatement
of the same SCF (oracle/oracle.py, pinned to fixtures made by running the
reference) -- with its matrix-free operator (oracle/fd_apply.c plus the
factored projectors, equal to the CSR product to rounding), numpy's global
seed 0, to the given tolerance.  It writes tests/golden/ref_<name>_tol<e>.json
and .npz in the layout of make_golden_configs.py, with "source" set to
"oracle".

The SCF fixed point does not depend on the Hartree solver (at convergence
the warm-started CG converges the potential either way); --cg_prec=1 reaches
it in fewer iterations (the oracle's spectral preconditioner) and keeps the
msecant1 mixer away from the history blow-ups a long plain-CG run meets at
this size.

Usage: python tests/golden/make_golden_oracle_configs.py NAME [--tol=1e-8] [--maxits=80] [--cg_prec=1]
"""
from __future__ import annotations

import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))


def main(name: str, tol: float, maxits: int, cg_prec: int = 0) -> None:
    from oracle import oracle as O
    from parsec_python_b200 import workloads as w

    cfg = w.config_system(name)
    dom = O.build_system(cfg["atoms"], h=cfg["h"], radius=cfg["radius"])
    tag = f"{name}_tol{int(round(-np.log10(tol)))}"
    np.random.seed(0)
    scf = O.OracleSCF(dom, cfg["atoms"], nev=cfg["nev"], poldeg=cfg["poldeg"], tol=tol, maxits=maxits,
                      operator="stencil", cg_prec=cg_prec)
    t0 = time.time()
    scf.setup()
    print(f"setup {scf.t_setup:.1f} s, n = {scf.n}", flush=True)
    while not scf.done():
        rec = scf.step()
        print(f"iter {rec['iter']:3d} err {rec['err']:.3e} E {rec['total_ry']:.10f} Ry  "
              f"cg {rec['cg_its']}  {rec['wall']:.1f} s", flush=True)
    wall = time.time() - t0
    res = scf.result()
    fin = res["energies"]
    hist = [r["total_ry"] for r in res["history"]]
    errs = [r["err"] for r in res["history"]]
    np.savez_compressed(HERE / f"ref_{tag}.npz", rho=res["rho"].astype(np.float32), eigenvalues=res["eigenvalues"],
                        occupations=res["occupations"], total_ry=np.array(fin["total_ry"]),
                        eigen_sum_ry=np.array(fin["eigen_sum_ry"]), hartree_ry=np.array(fin["hartree_ry"]),
                        xc_ry=np.array(fin["xc_ry"]), ion_ry=np.array(fin["ion_ry"]), log_total_ry=np.array(hist),
                        log_err=np.array(errs))
    meta = {"name": name, "source": "oracle", "operator": "stencil", "cg_prec": cg_prec, "domain": dom,
            "nev": cfg["nev"],
            "poldeg": cfg["poldeg"], "tol": tol, "seed": 0, "iterations": res["iterations"],
            "error": float(res["error"]), "converged": bool(res["converged"]), "wall_s": wall,
            "total_ry": fin["total_ry"], "cpu": os.cpu_count(),
            "iterations_to_1e-6": next((i + 1 for i, e in enumerate(errs) if e <= 1e-6), None),
            "log_err": errs}
    (HERE / f"ref_{tag}.json").write_text(json.dumps(meta, indent=1))
    print(json.dumps(meta), flush=True)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    opts = dict(a[2:].split("=", 1) for a in sys.argv[1:] if a.startswith("--") and "=" in a)
    if not args:
        sys.exit(f"usage: python {sys.argv[0]} NAME [--tol=1e-8] [--maxits=80]")
    main(args[0], float(opts.get("tol", 1e-8)), int(opts.get("maxits", 80)), int(opts.get("cg_prec", 0)))
