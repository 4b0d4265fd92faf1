"""The oracle's matrix-free operator (oracle/fd_apply.c + factored projectors)
against its CSR form, which the golden fixtures pin to the reference.

The large-configuration fixtures (tests/golden/make_golden_oracle_configs.py)
run the oracle with this operator, because the reference's CSR products take
minutes per block at 729,000 points.  These tests check that the operator is
the same matrix: every FD order, vectors and blocks in both memory orders,
with projectors and a local potential, to rounding; and that a short SCF
takes the same trajectory with either form."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O

A0 = O.A0_ANG


def _h2o():
    return [{"typ": "O", "coord": np.array([[0.0, 0.0, 0.0]]) / A0},
            {"typ": "H", "coord": np.array([[0.757, 0.586, 0.0], [-0.757, 0.586, 0.0]]) / A0}]


@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_stencil_operator_equals_csr(order):
    dom = {"nx": 22, "ny": 17, "nz": 13, "h": 0.4, "radius": 4.2}
    n = 22 * 17 * 13
    E, T = O.load_elements(), O.load_tables()
    atoms = _h2o()
    projs = O.projectors(dom, atoms, E, T)
    _, h0, pp, _ = O.pseudo_diag(dom, atoms, E, T)
    pot = pp + h0
    B = (0.5 * O.laplacian(dom, order) + O.nonlocal_csr(projs, n) + sp.diags(pot, 0, shape=(n, n))).tocsr()
    A = O.laplacian(dom, order)
    Hs, As = O.StencilHamiltonian(dom, order, projs, pot), O.StencilLaplacian(dom, order)
    rng = np.random.default_rng(order)
    for X in (rng.standard_normal(n), rng.standard_normal((n, 5)), np.asfortranarray(rng.standard_normal((n, 7))),
              rng.standard_normal((n, 1))):
        for op, ref in ((Hs, B), (As, A)):
            r, s = ref @ X, op @ X
            assert s.shape == r.shape
            assert np.abs(r - s).max() <= 1e-14 * np.abs(r).max()
        assert np.abs(As.dot(X) - A.dot(X)).max() <= 1e-14 * np.abs(A.dot(X)).max()


def test_stencil_operator_scf_follows_csr_scf():
    dom = O.build_system(_h2o(), h=0.5, radius=4.5)
    runs = {}
    for op in ("csr", "stencil"):
        np.random.seed(3)
        scf = O.OracleSCF(dom, _h2o(), nev=8, poldeg=8, tol=1e-6, maxits=4, operator=op)
        scf.setup()
        runs[op] = [scf.step() for _ in range(4)]
    for a, b in zip(runs["csr"], runs["stencil"]):
        assert abs(a["total_ry"] - b["total_ry"]) < 1e-9 * abs(a["total_ry"])
        assert np.abs(a["lam"] - b["lam"]).max() < 1e-9
        assert a["cg_its"] == b["cg_its"]


def test_operator_rejects_unknown_form():
    with pytest.raises(ValueError):
        O.OracleSCF({"nx": 4, "ny": 4, "nz": 4, "h": 1.0, "radius": 1.5}, _h2o(), nev=2, operator="dense")
