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


def test_hamiltonian_on_h2o_grid_matches_reference_csr(golden_dir, tables):
    """The oracle's B = 0.5 A + V_nl + diag(pot) on the H2O configuration's
    52^3 grid against the reference's assembled CSR applied to the same two
    seeded columns (tests/golden/make_golden_hx.py), CSR and matrix-free."""
    from parsec_python_b200 import workloads

    elements, tab = tables
    ref = np.load(golden_dir / "ref_hx_h2o.npz")
    cfg = workloads.config_system("h2o")
    dom = O.build_system(cfg["atoms"], h=cfg["h"], radius=cfg["radius"])
    n = dom["nx"] ** 3
    projs = O.projectors(dom, cfg["atoms"], elements, tab)
    B = (0.5 * O.laplacian(dom, 8) + O.nonlocal_csr(projs, n) + sp.diags(ref["pot"], 0, shape=(n, n))).tocsr()
    X = np.random.default_rng(11).standard_normal((n, 2))
    y = ref["y"]
    assert np.abs(B @ X - y).max() <= 1e-13 * np.abs(y).max()
    Hs = O.StencilHamiltonian(dom, 8, projs, ref["pot"])
    assert np.abs(Hs @ X - y).max() <= 1e-12 * np.abs(y).max()


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


@pytest.mark.parametrize("name,group_size", [("anderson", 0), ("group2", 2)])
def test_mixer2_bit_exact_including_restart(golden_dir, name, group_size):
    """Type-II multisecant mixer (Anderson for group_size 0) against the
    reference's own msecant2 outputs, through the restart at step 9 and the
    alternating EN stages after it (tests/golden/make_golden_mixer2.py)."""
    g = np.load(golden_dir / "ref_mixer2.npz")
    m = O.MSecant2(group_size=group_size)
    for i in range(len(g[f"{name}_x"])):
        out, used = m(g[f"{name}_x"][i], g[f"{name}_f"][i])
        assert used == int(g[f"{name}_m"][i])
        np.testing.assert_array_equal(out, g[f"{name}_out"][i])


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


# ---- Lanczos-based eigensolvers (diagmeth 0/1/2), tests/golden/make_golden_lanczos.py ----
H2O = [("O", [[0.0, 0.0, 0.0]]), ("H", [[0.757, 0.586, 0.0], [-0.757, 0.586, 0.0]])]


def _h2o_atoms():
    return [{"typ": t, "coord": np.array(c) / O.A0_ANG} for t, c in H2O]


@pytest.fixture(scope="module")
def lz(golden_dir):
    return np.load(golden_dir / "ref_lanczos.npz"), json.loads((golden_dir / "ref_lanczos.json").read_text())


def _hamiltonian(dom, tables, pot_ref):
    elements, tab = tables
    n = dom["nx"] ** 3
    rho0, hpot0, ppot, _ = O.pseudo_diag(dom, _h2o_atoms(), elements, tab)
    pot = ppot + hpot0
    np.testing.assert_array_equal(pot, pot_ref)
    vnl = O.nonlocal_csr(O.projectors(dom, _h2o_atoms(), elements, tab), n)
    return (0.5 * O.laplacian(dom, 8) + vnl + sp.diags(pot, 0, shape=(n, n))).tocsr()


@pytest.mark.parametrize("tag", ["small", "big"])
def test_lanczos_for_chsubsp_matches_reference(lz, tables, tag):
    """Both branches of lanczosForChsubsp: with the convergence test
    (n = 13824) and without it (n = 39304 > 35000)."""
    g, meta = lz
    dom = meta[tag]["domain"]
    B = _hamiltonian(dom, tables, g[f"{tag}_pot"])
    W, lam, bound = O.lanczos_for_chsubsp(B, 27, g[f"{tag}_v"].copy(), 450)
    assert np.abs(lam - g[f"{tag}_lfc_lam"]).max() < 1e-12
    assert abs(bound - float(g[f"{tag}_lfc_bound"])) < 1e-12 * abs(bound)
    assert np.abs((W[:, :4] ** 2).sum(1) - g[f"{tag}_lfc_rho4"]).max() < 1e-12


def test_chsubsp_and_lanczos_match_reference(lz, tables):
    g, meta = lz
    B = _hamiltonian(meta["small"]["domain"], tables, g["small_pot"])
    np.random.seed(meta["small"]["chsubsp_seed"])
    W, ritz = O.chsubsp(10, 27, B)
    assert np.abs(ritz - g["small_ch_ritz"]).max() < 1e-12
    assert np.abs((W[:, :4] ** 2).sum(1) - g["small_ch_rho4"]).max() < 1e-12
    # the CPU lanczos.py cannot run its own convergence test (n <= 35000)
    assert meta["small"]["lanczos_cpu"] != "ran"
    B = _hamiltonian(meta["big"]["domain"], tables, g["big_pot"])
    W, lam = O.lanczos(B, 27, g["big_lz_v"].copy(), 512, 1e-5)
    assert np.abs(lam - g["big_lz_lam"]).max() < 1e-12
    assert np.abs((W[:, :4] ** 2).sum(1) - g["big_lz_rho4"]).max() < 1e-12


def test_distinct_count_is_the_reference_pruning():
    """The greedy walk equals the reference's repeated np.delete pruning
    (lanczosForChsubsp.py:148-154) on sorted inputs with ties and chains."""
    rng = np.random.default_rng(5)
    for trial in range(200):
        base = np.sort(rng.uniform(-2, 2, rng.integers(1, 40)))
        rr = np.sort(np.concatenate([base, base[: rng.integers(0, len(base) + 1)] + rng.uniform(-2e-5, 2e-5)]))
        ref = rr.copy()
        c = 0
        while c < len(ref) - 1:
            ref = np.delete(ref, np.where(np.abs(ref[c] - ref[c + 1:]) < 1e-5)[0] + c + 1)
            c += 1
        assert O.distinct_count(rr) == len(ref)


def test_scf_diagmeth2_matches_reference(lz, tables):
    elements, tab = tables
    g, meta = lz
    ms = meta["scf_diagmeth2"]
    r = O.run_scf(ms["domain"], _h2o_atoms(), nev=12, poldeg=10, tol=1e-6, seed=0, elements=elements, tables=tab,
                  diagmeth=2)
    assert r["iterations"] == ms["iterations"]
    # 450 Lanczos steps without reorthogonalisation amplify the last-bit
    # differences of the sparse products (the oracle's CSR column order is not
    # the reference's), so the trajectory agrees to 1e-9 Ry here, not 1e-12
    assert abs(r["energies"]["total_ry"] - ms["total_ry"]) < 1e-8
    assert np.abs(r["eigenvalues"][:12] - g["scf2_eigenvalues"][:12]).max() < 1e-8


# ---- preconditioned CG (cg_prec = 1), tests/golden/make_golden_pcg_prec.py ----
def test_preconditioned_pcg_matches_reference(golden_dir):
    g = np.load(golden_dir / "ref_pcg_prec.npz")
    for tag in ("a", "b"):
        nx, ny, nz, order = (int(v) for v in g[f"{tag}_dims"])
        h = float(g[f"{tag}_h"])
        dom = {"nx": nx, "ny": ny, "nz": nz, "h": h}
        A = (1.0 / (h * h)) * O.fd3d(nx, ny, nz, order)
        x, its = O.pcg_prec(A, g[f"{tag}_rhs"], g[f"{tag}_x0"], 200, 1e-5, O.spectral_preconditioner(dom, order))
        assert its == int(g[f"{tag}_its"])
        np.testing.assert_allclose(x, g[f"{tag}_x"], rtol=0, atol=1e-12 * np.abs(g[f"{tag}_x"]).max())


def test_spectral_preconditioner_inverts_the_second_order_stencil():
    """For fd_order 2 the odd-reflected stencil is A itself: M = A^-1."""
    dom = {"nx": 9, "ny": 7, "nz": 8, "h": 0.5}
    A = O.laplacian(dom, 2)
    r = np.random.default_rng(3).standard_normal(9 * 7 * 8)
    z = O.spectral_preconditioner(dom, 2)(r)
    assert np.abs(A @ z - r).max() < 1e-12 * np.abs(r).max()


# ---- ML-grid density modes (sad_ml_grid, ml), tests/golden/make_golden_ml.py ----
ML_ATOMS = [("O", [[3.0, 3.0, 3.1]]), ("H", [[3.757, 3.586, 3.1], [2.243, 3.586, 3.1]])]


@pytest.fixture(scope="module")
def mlg(golden_dir):
    return np.load(golden_dir / "ref_ml.npz"), json.loads((golden_dir / "ref_ml.json").read_text())


def _ml_atoms():
    return [{"typ": t, "coord": np.array(c) / O.A0_ANG} for t, c in ML_ATOMS]


def test_ml_grid_setup_and_density_file_match_reference(mlg, tables):
    """pseudoDiag_MLgrid and pseudoDiag_ML4Den bit for bit, the ML-grid
    projectors to rounding."""
    elements, tab = tables
    g, meta = mlg
    dom = meta["domain"]
    r0, h0, p0, _ = O.pseudo_diag(O.ml_grid(dom), _ml_atoms(), elements, tab)
    assert (sha(r0), sha(h0), sha(p0)) == (meta["mlgrid"]["rho0"], meta["mlgrid"]["hpot0"], meta["mlgrid"]["ppot"])
    vnl = O.nonlocal_csr(O.projectors(O.ml_grid(dom), _ml_atoms(), elements, tab), dom["nx"] ** 3)
    assert np.abs(vnl @ g["vnl_x"] - g["vnl_y"]).max() <= 1e-12 * np.abs(g["vnl_y"]).max()
    r1, hp1, pp, info = O.ml_density_start(dom, _ml_atoms(), elements, tab, g["density"])
    assert sha(r1) == meta["ml4den"]["rho1"] and sha(pp) == meta["ml4den"]["pot"]
    assert np.abs(hp1 - g["ml_hpot1"]).max() <= 1e-12 * np.abs(g["ml_hpot1"]).max()
    assert info == meta["ml4den"]["info"]


@pytest.mark.parametrize("dm", ["sad_ml_grid", "ml"])
def test_ml_mode_scf_matches_reference(mlg, tables, dm):
    elements, tab = tables
    g, meta = mlg
    ms = meta[f"scf_{dm}"]
    r = O.run_scf(ms["domain"], _ml_atoms(), nev=12, poldeg=10, tol=1e-6, seed=0, elements=elements, tables=tab,
                  diagmeth=ms["diagmeth"], density_method=dm, density=g["density"], maxits=60)
    assert r["iterations"] == ms["iterations"]
    assert abs(r["energies"]["total_ry"] - ms["total_ry"]) < 1e-7
    assert np.abs(r["eigenvalues"][:12] - g[f"scf_{dm}_eigenvalues"][:12]).max() < 1e-8
