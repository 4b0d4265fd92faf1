"""The ML-grid density modes on the GPU (density_method = sad_ml_grid and ml)
against the reference's own outputs (tests/golden/make_golden_ml.py): the
ML-grid SAD setup and projector tables bit for bit, the density-file start,
and whole SCFs of both modes run from the reference-format input files
through the public entry point (1e-5 Ha bar)."""
import hashlib
import json
import shutil

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from parsec_python_b200 import gpu  # noqa: E402
from parsec_python_b200.__main__ import main as cli_main  # noqa: E402
from parsec_python_b200.inputs import ElementTable, pseudo_tables  # noqa: E402
from parsec_python_b200.models import A0_ANG  # noqa: E402

ML_ATOMS = [("O", [[3.0, 3.0, 3.1]]), ("H", [[3.757, 3.586, 3.1], [2.243, 3.586, 3.1]])]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def mlg(golden_dir):
    return np.load(golden_dir / "ref_ml.npz"), json.loads((golden_dir / "ref_ml.json").read_text())


def _atoms():
    return [{"typ": t, "coord": np.array(c) / A0_ANG} for t, c in ML_ATOMS]


def test_ml_grid_setup_bit_exact(mlg):
    g, meta = mlg
    ctx = gpu.GridContext(meta["domain"], 8)
    rho0, hpot0, ppot, info = gpu.sad_setup(ctx, _atoms(), ElementTable(), pseudo_tables(), ml_grid=True)
    assert sha(rho0.cpu().numpy()) == meta["mlgrid"]["rho0"]
    assert sha(hpot0.cpu().numpy()) == meta["mlgrid"]["hpot0"]
    assert sha(ppot.cpu().numpy()) == meta["mlgrid"]["ppot"]
    nl = gpu.projector_setup(ctx, _atoms(), ElementTable(), pseudo_tables(), ml_grid=True)
    ref = O.projectors(O.ml_grid(meta["domain"]), _atoms(), O.load_elements(), O.load_tables())
    off, idx, u, w = nl.tables()
    assert nl.n_atoms == len(ref)
    for a, pr in enumerate(ref):
        np.testing.assert_array_equal(idx[off[a]:off[a + 1]], pr["idx"])
        np.testing.assert_array_equal(u[:, off[a]:off[a + 1]], pr["u"])


def test_density_file_start_matches_reference(mlg, tmp_path):
    g, meta = mlg
    np.save(tmp_path / "d.npy", g["density"])
    ctx = gpu.GridContext(meta["domain"], 8)
    rho1, hpot1, ppot, info = gpu.ml_density_setup(ctx, _atoms(), ElementTable(), pseudo_tables(),
                                                   str(tmp_path / "d.npy"))
    assert sha(rho1.cpu().numpy()) == meta["ml4den"]["rho1"]
    assert sha(ppot.cpu().numpy()) == meta["ml4den"]["pot"]
    # the reference's 200-iteration CG from zero and ours differ by rounding
    ref = g["ml_hpot1"]
    assert np.abs(hpot1.cpu().numpy() - ref).max() <= 1e-8 * np.abs(ref).max()
    ri = meta["ml4den"]["info"]
    assert info["electron_count_initial"] == ri["electron_count_initial"]
    assert info["electron_count_normalized"] == ri["electron_count_normalized"]
    assert info["negative_values_zeroed"] == 4
    with pytest.raises(ValueError, match="does not match the grid"):
        np.save(tmp_path / "bad.npy", g["density"][:, :, :-1])
        gpu.ml_density_setup(ctx, _atoms(), ElementTable(), pseudo_tables(), str(tmp_path / "bad.npy"))


@pytest.mark.parametrize("dm", ["sad_ml_grid", "ml"])
def test_ml_mode_scf_from_input_file(mlg, golden_dir, tmp_path, dm):
    """python -m parsec_python_b200 on the reference-format .in (density file,
    POSCAR cell, diagmeth 2 by default) reaches the reference's energy."""
    g, meta = mlg
    for f in ("cell.POSCAR", "density.npy", f"h2o_{dm}.in"):
        shutil.copy(golden_dir / "ml" / f, tmp_path / f)
    res = cli_main([str(tmp_path / f"h2o_{dm}.in")])
    ms = meta[f"scf_{dm}"]
    assert res.converged
    assert abs(res.history[-1]["total_ry"] - ms["total_ry"]) < 2e-5
    assert np.abs(res.eigenvalues[:12] - g[f"scf_{dm}_eigenvalues"][:12]).max() < 1e-5
    h = ms["domain"]["h"]
    assert np.abs(res.rho.cpu().numpy() - g[f"scf_{dm}_rho"]).sum() * h ** 3 < 1e-4
    out = (tmp_path / f"h2o_{dm}.out").read_text()
    assert f"Density initialization: {dm}" in out
    assert "chsubsp" in out
