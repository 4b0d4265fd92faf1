"""Pin the CPU oracle to outputs of the reference itself (tests/golden/,
written by tests/golden/make_golden.py from PARSEC.py's own CPU code)."""
import hashlib
import json

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def meta(golden_dir):
    return json.loads((golden_dir / "ref_meta.json").read_text())


@pytest.fixture(scope="module")
def tables():
    return O.load_elements(), O.load_tables()


def _atoms(spec):
    return [{"typ": t, "coord": np.array(c, dtype=np.float64)} for t, c in spec]


def test_element_table_matches_reference_parse(meta, tables):
    elements, _ = tables
    for el, (z, zv, h, r, big_r) in meta["elements"].items():
        e = elements[el]
        assert (e["Z"], e["Zvalue"], e["h"], e["r"], e["R"]) == (z, zv, h, r, big_r)


def test_fd3d_bit_exact(golden_dir):
    fd = np.load(golden_dir / "ref_fd3d.npz")
    for k in fd.files:
        if k.startswith("x_"):
            nx, ny, nz, order = map(int, k[2:].split("_"))
            y = O.fd3d(nx, ny, nz, order) @ fd[k]
            np.testing.assert_array_equal(y, fd["y_" + k[2:]], err_msg=k)


def test_splines_bit_exact(golden_dir, meta, tables):
    _, tab = tables
    spl = np.load(golden_dir / "ref_splines.npz")
    for tag, m in meta["splines"].items():
        el, name = tag.split("_", 1)
        d = tab[el]
        y = {"charge": d[:, 1], "hartree": d[:, 2], "pot_S": d[:, 4], "wfn_P": d[:, 5],
             "potPS": d[:, 3] - d[:, 4]}[name]
        keep = O.prune_knots(y)
        s = O.Spline(d[keep, 0], y[keep])
        assert sha(keep.astype(np.int64)) == m["keep"], tag
        assert (sha(s.z), sha(s.c), sha(s.d)) == (m["z"], m["c"], m["d"]), tag
        np.testing.assert_array_equal(s(spl["r_" + tag]), spl["v_" + tag], err_msg=tag)


def test_pseudo_diag_and_projectors(golden_dir, meta, tables):
    elements, tab = tables
    ion = np.load(golden_dir / "ref_ion_h2o.npz")
    mi = meta["ion_h2o"]
    atoms = _atoms(mi["atoms"])
    rho0, hpot0, ppot, info = O.pseudo_diag(mi["domain"], atoms, elements, tab)
    assert (sha(rho0), sha(hpot0), sha(ppot)) == (mi["rho0"], mi["hpot0"], mi["ppot"])
    assert info["electron_count_initial"] == mi["info"]["electron_count_initial"]
    projs = O.projectors(mi["domain"], atoms, elements, tab)
    n = mi["domain"]["nx"] ** 3
    np.testing.assert_array_equal(O.nonlocal_csr(projs, n) @ ion["vnl_x"], ion["vnl_y"])
    yf = O.nonlocal_apply(projs, ion["vnl_x"])
    assert np.abs(yf - ion["vnl_y"]).max() <= 1e-13 * np.abs(ion["vnl_y"]).max()
    assert O.nuclear(atoms, elements) == mi["e_nuc"]


def test_sample_h2o_sad_density_bit_exact(meta, tables):
    """Known-answer test: the shipped samples/h2o/*_init_rho_grid.npy."""
    elements, tab = tables
    f = 1.0 / O.A0_ANG
    o = np.array([[-3.56626, 1.77639, 0.0]]) * f
    hh = np.array([[-2.59626, 1.77639, 0.0], [-3.88959, 1.36040, -0.81444]]) * f
    c = np.mean(np.vstack([o, hh]), axis=0)
    atoms = [{"typ": "O", "coord": o - c}, {"typ": "H", "coord": hh - c}]
    dom = O.build_system(atoms, h=0.2 * f, radius=5.0 * f)
    assert dom["nx"] == 52
    rho0 = O.pseudo_diag(dom, atoms, elements, tab)[0]
    grid = rho0.reshape((dom["nx"], dom["ny"], dom["nz"]), order="F")
    assert sha(grid) == meta["sample_h2o_init_rho_grid"]["sha256"]


def test_xc(golden_dir):
    xc = np.load(golden_dir / "ref_xc.npz")
    v, e = O.exc_nspn(0.37, xc["rho"])
    assert np.abs(v - xc["vxc"]).max() <= 1e-14 * np.abs(xc["vxc"]).max()
    assert abs(e - float(xc["exc"])) <= 1e-13 * abs(float(xc["exc"]))


def test_mixer_bit_exact_including_restart(golden_dir):
    mx = np.load(golden_dir / "ref_mixer.npz")
    m = O.MSecant1()
    restarted = False
    for i in range(len(mx["x"])):
        before = 0 if m.DX is None else m.DX.shape[1]
        out, used = m(mx["x"][i], mx["f"][i])
        restarted |= before >= 2 and used == 0
        np.testing.assert_array_equal(out, mx["out"][i])
    assert restarted


def test_occupations_bit_exact(golden_dir):
    oc = np.load(golden_dir / "ref_occupations.npz")
    for i in range(4):
        c, occ = O.occupations(oc[f"lam_{i}"], 500.0, int(oc[f"ne_{i}"]), 1e-6)
        assert c == float(oc[f"ef_{i}"])
        np.testing.assert_array_equal(occ, oc[f"occ_{i}"])


def test_pcg_bit_exact(golden_dir):
    pc = np.load(golden_dir / "ref_pcg.npz")
    A = (1.0 / (0.4 * 0.4)) * O.fd3d(10, 10, 10, 8)
    x, its = O.pcg(A, pc["rhs"], pc["x0"], 200, 1e-5)
    assert its == int(pc["its"])
    np.testing.assert_array_equal(x, pc["x"])


def test_lanczos_and_filters(golden_dir, meta, tables):
    elements, tab = tables
    ev = np.load(golden_dir / "ref_eigs.npz")
    mi = meta["ion_h2o"]
    dom = mi["domain"]
    n = dom["nx"] ** 3
    atoms = _atoms(mi["atoms"])
    vnl = O.nonlocal_csr(O.projectors(dom, atoms, elements, tab), n)
    B = (0.5 * O.laplacian(dom, 8) + vnl + sp.diags(ev["pot"], 0, shape=(n, n))).tocsr()
    np.random.seed(7)
    ub, ritz = O.lancz_uppbnd(n, B)
    assert abs(ub - float(ev["uppbnd"])) <= 1e-13 * abs(ub)
    np.random.seed(8)
    assert abs(O.lanczos_bound(B, np.random.randn(n, 1)) - float(ev["bound"])) <= 1e-13 * abs(ub)
    np.random.seed(9)
    W, lam = O.first_filt(27, B, 10)
    assert np.abs(lam - ev["ff_lam"]).max() < 1e-12
    np.random.seed(10)
    W2, lam2 = O.chefsi1(W, lam, 10, 12, B)
    assert np.abs(lam2 - ev["cf_lam"]).max() < 1e-12
    assert np.abs((W2[:, :12] ** 2).sum(1) - ev["cf_rho"]).max() < 1e-12


def test_scf_h2o_small_matches_reference(golden_dir, meta, tables):
    elements, tab = tables
    sc = np.load(golden_dir / "ref_scf_h2o.npz")
    ms = meta["scf_h2o"]
    atoms = [{"typ": "O", "coord": np.array([[0.0, 0.0, 0.0]]) / O.A0_ANG},
             {"typ": "H", "coord": np.array([[0.757, 0.586, 0.0], [-0.757, 0.586, 0.0]]) / O.A0_ANG}]
    r = O.run_scf(ms["domain"], atoms, nev=12, poldeg=10, tol=1e-6, seed=0, elements=elements, tables=tab)
    assert r["iterations"] == ms["iterations"]
    assert abs(r["energies"]["total_ry"] - ms["total_ry"]) < 1e-10
    assert np.abs(r["eigenvalues"] - sc["eigenvalues"]).max() < 1e-10
    h = ms["domain"]["h"]
    assert np.abs(r["rho"] - sc["rho"]).sum() * h ** 3 < 1e-9
