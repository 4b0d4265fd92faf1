"""Whole-SCF parity on the GPU against the reference's own SCF results.

The bar: total energy and
eigenvalues within 1e-5 Ha of the reference CPU path on the same input,
integrated |delta rho| within 1e-4 electrons.  Energies are compared in Ry
(1e-5 Ha = 2e-5 Ry).  The GPU and the reference draw different random
starting vectors, so agreement is that of converged fixed points."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from parsec_python_b200 import workloads  # noqa: E402
from parsec_python_b200.backend import select_solver_backend  # noqa: E402
from parsec_python_b200.inputs import ElementTable  # noqa: E402
from parsec_python_b200.models import A0_ANG, SolverSettings  # noqa: E402
from parsec_python_b200.solver import run_rsdft_calculation  # noqa: E402
from parsec_python_b200.system import system_from_atoms  # noqa: E402

HA = 2.0  # Ry per Ha
E_TOL_RY = 1e-5 * HA
RHO_TOL = 1e-4


def run_gpu(atoms_bohr, h, radius, nev, poldeg, tol, precision="fp64", seed=0, maxits=60):
    s = SolverSettings(tol=tol, poldeg=poldeg, maxits=maxits, precision=precision, seed=seed)
    s.normalize()
    elem = ElementTable()
    prob = system_from_atoms(atoms_bohr, h=h, radius=radius, nev=nev, settings=s, elem=elem)
    backend = select_solver_backend(s)
    return prob, run_rsdft_calculation(prob, elem, len(elem), backend, verbose=False)


def occupied(ref, nev):
    """States the reference occupies (f > 1e-6): their eigenvalues converge
    with the density.  The empty states at the top of the nev window converge
    only as fast as the filter reaches them, differently in every run."""
    return int(np.count_nonzero(np.asarray(ref["occupations"])[:nev] > 1e-6))


def check(prob, res, ref, nev):
    h = prob.domain["h"]
    e = res.history[-1]["total_ry"]
    assert res.converged
    assert abs(e - float(ref["total_ry"])) < E_TOL_RY, (e, float(ref["total_ry"]))
    nocc = occupied(ref, nev)
    assert np.abs(res.eigenvalues[:nocc] - ref["eigenvalues"][:nocc]).max() < 1e-5
    drho = np.abs(res.rho.cpu().numpy() - ref["rho"].astype(np.float64)).sum() * h ** 3
    assert drho < RHO_TOL, drho
    return e, drho


def test_scf_small_h2o_matches_reference(golden_dir):
    meta = json.loads((golden_dir / "ref_meta.json").read_text())["scf_h2o"]
    ref = np.load(golden_dir / "ref_scf_h2o.npz")
    atoms = [{"typ": "O", "coord": np.array([[0.0, 0.0, 0.0]]) / A0_ANG},
             {"typ": "H", "coord": np.array([[0.757, 0.586, 0.0], [-0.757, 0.586, 0.0]]) / A0_ANG}]
    dom = meta["domain"]
    prob, res = run_gpu(atoms, dom["h"], 4.0 / A0_ANG, 12, 10, 1e-6)
    assert prob.domain == dom
    check(prob, res, ref, 12)
    # the reference's iteration count at the same tolerance, within a couple
    assert abs(res.iterations - meta["iterations"]) <= 3


def test_scf_is_deterministic():
    atoms = workloads.to_bohr(workloads.h2o())
    _, a = run_gpu(atoms, 0.3 / A0_ANG, 4.0 / A0_ANG, 12, 10, 1e-6, seed=5)
    _, b = run_gpu(atoms, 0.3 / A0_ANG, 4.0 / A0_ANG, 12, 10, 1e-6, seed=5)
    assert a.iterations == b.iterations
    assert a.history[-1]["total_ry"] == b.history[-1]["total_ry"]
    assert torch.equal(a.rho, b.rho)


# H2O converges to the same fixed point at the configuration's tol 1e-6 (the
# reference's own seed-to-seed spread there is ~1e-6 Ha).  For C10H8 the
# reference's seed-to-seed spread at tol 1e-6 is 2.2e-5 Ha, above the bar, so
# both sides are compared at tol 1e-8; likewise Si35H36 (the reference's own
# SCF) and Si87H76 (the oracle with its matrix-free operator: the reference's
# CSR SCF would take many hours at 729,000 points and 292 states).
@pytest.mark.parametrize("name,tag", [("h2o", "h2o"), ("c10h8", "c10h8_tol8"), ("si35h36", "si35h36_tol8"),
                                      ("si87h76", "si87h76_tol8")])
def test_benchmark_config_matches_reference(golden_dir, name, tag):
    f = golden_dir / f"ref_{tag}.npz"
    if not f.exists():
        pytest.skip(f"{f.name} not generated")
    meta = json.loads((golden_dir / f"ref_{tag}.json").read_text())
    ref = np.load(f)
    cfg = workloads.config_system(name)
    prob, res = run_gpu(cfg["atoms"], cfg["h"], cfg["radius"], cfg["nev"], cfg["poldeg"], meta["tol"], maxits=80)
    assert prob.domain["nx"] == meta["domain"]["nx"]
    check(prob, res, ref, cfg["nev"])


@pytest.mark.parametrize("group_size", [0, 2], ids=["anderson", "groups-of-2"])
def test_scf_with_type2_mixer_lands_on_the_reference(golden_dir, group_size):
    """The Type-II multisecant mixer (Mixer/msecant2.py; group size 0 is the
    Anderson mixing the H2O configuration names) on the H2O configuration:
    the converged fixed point does not depend on the mixer, so the same
    energy, eigenvalue and density bars hold against the reference's SCF."""
    meta = json.loads((golden_dir / "ref_h2o.json").read_text())
    ref = np.load(golden_dir / "ref_h2o.npz")
    cfg = workloads.config_system("h2o")
    s = SolverSettings(tol=meta["tol"], poldeg=cfg["poldeg"], maxits=80, mixer="msecant2",
                       mix_group_size=group_size)
    s.normalize()
    elem = ElementTable()
    prob = system_from_atoms(cfg["atoms"], h=cfg["h"], radius=cfg["radius"], nev=cfg["nev"], settings=s, elem=elem)
    res = run_rsdft_calculation(prob, elem, len(elem), select_solver_backend(s), verbose=False)
    print(f"msecant2 group size {group_size}: {res.iterations} iterations (reference msecant1: "
          f"{meta.get('iterations')}); errors", " ".join(f"{r['err']:.1e}" for r in res.history))
    check(prob, res, ref, cfg["nev"])


def _mixed_vs_reference(golden_dir, name, tag, switch):
    f = golden_dir / f"ref_{tag}.npz"
    if not f.exists():
        pytest.skip(f"{f.name} not generated")
    ref = np.load(f)
    cfg = workloads.config_system(name)
    s = SolverSettings(tol=1e-8, poldeg=cfg["poldeg"], maxits=80, precision="mixed", cg_prec=1, seed=2)
    s.mixed_switch = switch
    s.normalize()
    elem = ElementTable()
    prob = system_from_atoms(cfg["atoms"], h=cfg["h"], radius=cfg["radius"], nev=cfg["nev"], settings=s, elem=elem)
    res = run_rsdft_calculation(prob, elem, len(elem), select_solver_backend(s), verbose=False)
    nev, h = cfg["nev"], prob.domain["h"]
    nocc = occupied(ref, nev)
    de_ha = abs(res.history[-1]["total_ry"] - float(ref["total_ry"])) / HA
    dlam_ha = float(np.abs(res.eigenvalues[:nocc] - ref["eigenvalues"][:nocc]).max())
    drho = float(np.abs(res.rho.cpu().numpy() - ref["rho"].astype(np.float64)).sum() * h ** 3)
    f32_its = sum(1 for r in res.history if r["block_dtype"] == "f32")
    late = sum(1 for r in res.history if r["block_dtype"] == "f32" and r["late"])
    print(f"{name} mixed (switch {switch}): {res.iterations} its ({f32_its} FP32, {late} of them late), "
          f"|dE| {de_ha:.2e} Ha, "
          f"max |d lambda| (occupied) {dlam_ha:.2e} Ha, int |d rho| {drho:.2e} e")
    return res, de_ha, dlam_ha, drho


@pytest.mark.parametrize("name,tag", [("si35h36", "si35h36_tol8"), ("si87h76", "si87h76_tol8")])
def test_mixed_precision_matches_reference(golden_dir, name, tag):
    """The chosen form (FP32 filter and tensor-core Rayleigh-Ritz products;
    below an SCF error of 1e-4 the round-to-nearest block product, below 1e-6
    FP64 blocks; preconditioned Hartree solve) driven to tol 1e-8 reaches the
    reference's FP64 fixed point: energy and every occupied eigenvalue within
    1e-5 Ha, integrated |delta rho| within 1e-4 e."""
    res, de, dlam, drho = _mixed_vs_reference(golden_dir, name, tag, 1e-4)
    assert res.converged
    assert de < 1e-5 and dlam < 1e-5 and drho < RHO_TOL


@pytest.mark.parametrize("name,tag", [("si35h36", "si35h36_tol8"), ("si87h76", "si87h76_tol8")])
def test_mixed_fp32_finish_lands_on_the_reference(golden_dir, name, tag):
    """The FP32 phases alone (mixed_finish = fp32): 30 iterations toward tol
    1e-8, below the FP32 floor of the SCF error, so the run ends on FP32
    iterations.  With the late phase's FP64-accumulated Gram pair and block
    product the FP32 fixed point is the reference's: integrated |delta rho|
    within 1e-4 e and every occupied eigenvalue within 1e-5 Ha; the energy
    (which the FP32 rounding moves by about 1e-5 Ha from one iteration to the
    next at the floor) within 5e-5 Ha."""
    f = golden_dir / f"ref_{tag}.npz"
    if not f.exists():
        pytest.skip(f"{f.name} not generated")
    ref = np.load(f)
    cfg = workloads.config_system(name)
    s = SolverSettings(tol=1e-8, poldeg=cfg["poldeg"], maxits=30, precision="mixed", cg_prec=1, seed=2,
                       mixed_finish="fp32")
    s.normalize()
    elem = ElementTable()
    prob = system_from_atoms(cfg["atoms"], h=cfg["h"], radius=cfg["radius"], nev=cfg["nev"], settings=s, elem=elem)
    res = run_rsdft_calculation(prob, elem, len(elem), select_solver_backend(s), verbose=False)
    assert all(r["block_dtype"] == "f32" for r in res.history)
    nev, h = cfg["nev"], prob.domain["h"]
    nocc = occupied(ref, nev)
    de_ha = abs(res.history[-1]["total_ry"] - float(ref["total_ry"])) / HA
    dlam_ha = float(np.abs(res.eigenvalues[:nocc] - ref["eigenvalues"][:nocc]).max())
    drho = float(np.abs(res.rho.cpu().numpy() - ref["rho"].astype(np.float64)).sum() * h ** 3)
    late = sum(1 for r in res.history if r["late"])
    print(f"{name} mixed, FP32 finish: {res.iterations} its ({late} late), error {res.history[-1]['err']:.1e}, "
          f"|dE| {de_ha:.2e} Ha, max |d lambda| (occupied) {dlam_ha:.2e} Ha, int |d rho| {drho:.2e} e")
    assert drho < RHO_TOL and dlam_ha < 1e-5 and de_ha < 5e-5
