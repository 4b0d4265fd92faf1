"""Host-side logic (no GPU): input parsing, units, system preparation,
settings overrides, output formats, benchmark geometries."""
import numpy as np
import pytest

from oracle import oracle as O
from parsec_python_b200 import workloads
from parsec_python_b200.inputs import ElementTable, load_atomic_data_from_file, prepare_input_data
from parsec_python_b200.models import SolverSettings
from parsec_python_b200 import output
from parsec_python_b200.system import prepare_system

SAMPLE_IN = """$system
O  -3.56626  1.77639  0.00000
H  -2.59626  1.77639  0.00000
H  -3.88959  1.36040 -0.81444
$system

$settings
unit = Angstrom
Z_charge = 0
density_method = sad
grid_spacing = 0.200000
sphere_radius = 5.000000
tol = 2.000000e-04
Fermi_temp = 500
maxits = 50
fd_order = 8
poldeg = 10
diagmeth = 3
save_wfn = 0
use_gpu = 0
recenter_atoms = 1
$settings
"""


def test_sample_input_prepares_the_reference_domain(tmp_path):
    f = tmp_path / "H2O_sad_diagmeth3_5A_0p2A.in"
    f.write_text(SAMPLE_IN)
    s = SolverSettings()
    data = prepare_input_data(s, str(f))
    s.apply_overrides(data.settings_overrides)
    assert (s.tol, s.maxits, s.poldeg, s.fd_order, s.diagmeth) == (2e-4, 50, 10, 8, 3)
    elem = ElementTable()
    p = prepare_system(data, s, elem)
    # values printed in the shipped samples/h2o/*.out
    assert p.domain["nx"] == 52 and p.nev == 16
    assert f"{p.domain['radius']:10.5f}" == "   9.63760"
    assert f"{p.h:10.5f}" == "   0.37795"
    c = np.vstack([a["coord"] for a in p.input_data.atoms])
    assert f"{c[0, 0]:12.6f}" == "   -0.407343" and f"{c[2, 2]:12.6f}" == "   -1.026046"
    assert p.paths.output_file.endswith("H2O_sad_diagmeth3_5A_0p2A.out")


def test_settings_override_rules():
    s = SolverSettings()
    ap = s.apply_overrides({"TOL": "6", "Fermi_temp": "300", "adaptiveScheme": "1", "unknown": 3, "write_wfn": "yes"})
    assert s.tol == 1e-6 and s.fermi_temp == 300.0 and s.adaptive_scheme == 1 and s.save_wfn == 1
    assert "unknown" not in ap
    s.apply_overrides({"diagmeth": 7})
    assert s.diagmeth == 3


def test_json_and_txt_inputs(tmp_path):
    j = tmp_path / "h.json"
    j.write_text('{"atoms": [{"typ": "H", "coord": [[0.0, 0.0, 0.0]]}], "charge": 0.0, '
                 '"settings": {"unit": "bohr", "maxits": 1, "nev": 1}}')
    d = load_atomic_data_from_file(str(j))
    assert d.atoms[0]["typ"] == "H" and d.settings_overrides["nev"] == 1 and d.settings_overrides["unit"] == "bohr"
    t = tmp_path / "x.txt"
    t.write_text("C 0 0 0\nH 1 0 0\nC 2 0 0\n")
    d = load_atomic_data_from_file(str(t))
    assert [a["typ"] for a in d.atoms] == ["C", "H"] and d.n_atom == [2, 1]
    with pytest.raises(ValueError):
        t.write_text("C 0 0\n")
        load_atomic_data_from_file(str(t))


def test_scf_iteration_block_format(tmp_path):
    from parsec_python_b200.models import EnergyComponents

    out = tmp_path / "a.out"
    output.initialize_output_file(str(out), "gpu", "sad")
    e = EnergyComponents(-10.78258, 45.85619, -8.79420, 13.76119, -40.14373)
    output.write_scf_iteration(str(out), 1, "first_filt_gpu (diagmeth=3)", 0.5, 2, np.array([-1.09310376, -0.65923964]),
                               np.array([1.0, 1.0]), 1e-5, "no prec", 0.1, 0.328, e, 3)
    text = out.read_text()
    assert "    1     -2.1862075200" in text
    assert "   ... SCF error =   3.28e-01" in text
    assert "     Total electronic energy = -546.18347  eV   =  -40.14373  Ry  " in text


def test_density_npy_variants(tmp_path):
    dom = {"nx": 4, "ny": 4, "nz": 4, "h": 0.5, "radius": 0.75}
    g = np.arange(64, dtype=float)
    output.save_density_variants(g, dom, str(tmp_path / "r"))
    a = np.load(tmp_path / "r_grid.npy")
    assert a.shape == (4, 4, 4) and a[1, 0, 0] == 1.0 and a[0, 1, 0] == 4.0
    np.testing.assert_allclose(np.load(tmp_path / "r_bohr3.npy"), a / 0.125)


def test_benchmark_geometries():
    c = workloads.count
    assert c(workloads.naphthalene()) == {"C": 10, "H": 8}
    assert c(workloads.sih_cluster(4)) == {"Si": 35, "H": 36}
    assert c(workloads.sih_cluster(7)) == {"Si": 87, "H": 76}
    for seed in (0, 5, 511):
        w = workloads.water_cluster(seed)
        n = c(w)["O"]
        assert 2 <= n <= 8 and c(w)["H"] == 2 * n
        o = w[0]["coord"]
        d = np.linalg.norm(o[:, None] - o[None], axis=-1) + np.eye(n) * 10
        assert d.min() >= 2.6 and np.linalg.norm(o, axis=1).max() <= 6.0


def test_oracle_and_product_grid_rules_agree():
    s = SolverSettings()
    elem = ElementTable()
    from parsec_python_b200.system import cube_for_radius

    for h, r in ((0.378, 9.45), (0.34, 13.2), (0.4724, 17.0)):
        assert cube_for_radius(r, h) == O.build_system([], h=h, radius=r)
    assert s.precision == "fp64" and len(elem) == 18


def test_learned_network_layout():
    """Channel bookkeeping of the encoder-decoder: every layer reads the
    channels its sources produce; about 1.3 M parameters."""
    from parsec_python_b200 import learned

    cout = {"in": 8}
    for l in learned.LAYERS:
        assert l.ca == cout[l.src], l.name
        assert l.cs == (cout[l.skip] if l.skip else 0), l.name
        assert l.ca % 8 == 0 and l.cs % 8 == 0 and l.cout % 8 == 0
        assert not (l.up and l.stride != 1)
        cout[l.name] = l.cout
    assert 1.2e6 < learned.n_params() < 1.4e6
    w = learned.load_weights()
    if w is not None:
        assert w["w"].size == learned.n_params()
        assert w["a0"] > 0 and w["a1"] > 0 and w["at"] > 0


def test_ml_density_inputs_read_grid_from_files(golden_dir):
    """The ML density modes take the grid from the density file's shape and the
    POSCAR cell (rsdft_input.py:560-579, rsdft_setup.py:40-63,106-117), keep
    the atoms in the cell frame and default to diagmeth 2 (main_new.py:76-78)."""
    import json

    from parsec_python_b200.inputs import ElementTable, has_diagmeth_override, prepare_input_data
    from parsec_python_b200.models import SolverSettings
    from parsec_python_b200.system import prepare_system

    meta = json.loads((golden_dir / "ref_ml.json").read_text())
    for dm in ("ml", "sad_ml_grid"):
        s = SolverSettings()
        s.normalize()
        data = prepare_input_data(s, str(golden_dir / "ml" / f"h2o_{dm}.in"))
        assert data.density_method == dm and data.grid_mode == "ml"
        assert data.ml_file_path.endswith("density.npy") and data.grid_poscar_path.endswith("cell.POSCAR")
        assert not has_diagmeth_override(data.settings_overrides)
        s.apply_overrides(data.settings_overrides)
        prob = prepare_system(data, s, ElementTable())
        ref = meta[f"scf_{dm}"]["domain"]
        assert prob.domain == pytest.approx(ref)
        assert prob.nev == meta[f"scf_{dm}"]["nev"]
        # no recentring on an ML grid: the oxygen stays at its cell position
        assert np.allclose(prob.input_data.atoms[0]["coord"], np.array([[3.0, 3.0, 3.1]]) / 0.529177210903)


def test_wfn_dat_round_trip(tmp_path):
    """load_wavefunction reads back what save_wavefunction writes (the
    reference's layout, rsdft_output.py:298-334), field by field."""
    rng = np.random.default_rng(2)
    n, nev = 300, 5
    dom = {"radius": 4.25, "h": 0.35, "nx": 7, "ny": 7, "nz": 7}
    pot, rho, W = rng.standard_normal(n), rng.random(n), rng.standard_normal((n, nev + 3))
    atoms = [{"typ": "O", "coord": rng.standard_normal((1, 3))}, {"typ": "H", "coord": rng.standard_normal((2, 3))}]
    f = tmp_path / "x_wfn.dat"
    output.save_wavefunction(str(f), dom, pot, rho, W, nev, 2, atoms)
    d = output.load_wavefunction(str(f))
    assert (d["radius"], d["h"], d["nev"]) == (4.25, 0.35, nev)
    np.testing.assert_array_equal(d["potential"], pot)
    np.testing.assert_array_equal(d["rho"], rho)
    np.testing.assert_array_equal(d["wavefunctions"], W[:, :nev])
    for a, b in zip(d["atoms"], atoms):
        np.testing.assert_array_equal(a, b["coord"])
    f.write_bytes(f.read_bytes() + b"x")
    with pytest.raises(ValueError, match="trailing"):
        output.load_wavefunction(str(f))


@pytest.mark.parametrize("kind", ["random", "graded", "steep", "dependent", "zero"])
def test_quasi_inverse_from_gram_matches_pivoted_qr(kind):
    """The Type-II mixer's quasi-inverse product C = qinv(A) qinv(A)^T
    (Mixer/qinv.py:5-62, pivoted QR of the n x r history block) computed from
    the r x r Gram matrix by a pivoted Cholesky, as the GPU mixer does: the
    same rank cut and C to 1e-10 on well-conditioned and graded blocks
    (column norms over six and over eighteen decades, as the newest residual
    differences of a converging SCF are: small columns are kept), and an
    exactly dependent or zero column dropped as the QR drops it."""
    from parsec_python_b200 import gpu

    rng = np.random.default_rng({"random": 1, "graded": 2, "steep": 5, "dependent": 3, "zero": 4}[kind])
    A = rng.standard_normal((300, 7))
    if kind == "graded":
        A *= 10.0 ** -np.arange(7)
    elif kind == "steep":
        A *= 10.0 ** (-3 * np.arange(7))
    elif kind == "dependent":
        A[:, 4] = A[:, 1]
    elif kind == "zero":
        A[:, 2] = 0.0
    B = O.qinv(A)
    ref = B @ B.T
    got = gpu.qinv_from_gram(A.T @ A, np.finfo(float).eps * np.linalg.norm(A, np.inf))
    # each entry against the scale of its columns (C_ij ~ 1 / (|a_i| |a_j|))
    cn = np.linalg.norm(A, axis=0)
    sc = np.where(np.outer(cn, cn) > 0, 1.0 / np.maximum(np.outer(cn, cn), 1e-300), 0.0)
    assert (np.abs(got - ref) <= 1e-9 * sc + 1e-12 * np.abs(ref).max()).all()
    assert ((got != 0) == (ref != 0)).all()


def test_input_file_selects_the_anderson_mixer(tmp_path):
    """`mixer = anderson` in the settings block of an .in file (a key of this
    library; the reference has no mixer key) reaches the solver settings."""
    f = tmp_path / "h2o_anderson.in"
    f.write_text(SAMPLE_IN.replace("diagmeth = 3", "diagmeth = 3\nmixer = anderson"))
    assert "mixer = anderson" in f.read_text()
    s = SolverSettings()
    data = prepare_input_data(s, str(f))
    s.apply_overrides(data.settings_overrides)
    s.normalize()
    assert (s.mixer, s.mix_group_size) == ("msecant2", 0)


def test_settings_select_the_anderson_mixer():
    s = SolverSettings()
    assert s.mixer == "msecant1"
    s.apply_overrides({"mixer": "anderson"})
    s.normalize()
    assert (s.mixer, s.mix_group_size) == ("msecant2", 0)
    s.apply_overrides({"mixer": "msecant2", "mix_group_size": "3"})
    s.normalize()
    assert (s.mixer, s.mix_group_size) == ("msecant2", 3)
    s.apply_overrides({"mixer": "nonsense"})
    s.normalize()
    assert s.mixer == "msecant1"
