"""Host control flow of the Type-II multisecant mixer (gpu.Mixer2), on CPU.

gpu.Mixer2 keeps its history in device memory and runs the control flow of
Mixer/msecant2.py on the host: the restart test, the alternating EN stages
after a restart, the groups and the quasi-inverse of the last group.  Here it
runs on CPU tensors with a stand-in context whose `call` carries out each
libpsc entry point it uses (psc_mix2_diff, psc_mix2_store, psc_block_dots,
psc_block_combine, psc_block_absrow_max, psc_dot, psc_gram, psc_gemm_nn) with
NumPy on the same memory, as the C ABI documents them.  So these tests check
the host logic -- which columns each call reads and writes, in which order --
against the oracle's msecant2 and the reference's own outputs; the GPU tests
check the kernels.
"""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O
from parsec_python_b200 import gpu
from parsec_python_b200._lib import F64


def _arr(p, count):
    """The `count` doubles at the address a c_void_p (from gpu._p) holds."""
    return np.ctypeslib.as_array((ctypes.c_double * count).from_address(p.value))


class HostContext:
    """The entry points gpu.Mixer2 calls, on host memory."""

    def __init__(self, n):
        self.n = n
        self.device = torch.device("cpu")

    def empty(self, *shape, dtype=torch.float64):
        return torch.empty(*shape, dtype=dtype)

    def call(self, name, *a):
        n = self.n
        if name == "psc_mix2_diff":
            x1, f1, dx, df = (_arr(p, n) for p in a[:4])
            df[:] = f1 - df
            dx[:] = (x1 - dx) + a[4] * df
        elif name == "psc_mix2_store":
            x1, f1, dx, df = (_arr(p, n) for p in a[:4])
            dx[:] = x1
            df[:] = f1
        elif name == "psc_dot":
            _arr(a[3], 1)[0] = _arr(a[0], a[2]) @ _arr(a[1], a[2])
        elif name == "psc_block_dots":
            A, lda, r, x, out = a[:5]
            if r:
                _arr(out, r)[:] = _arr(A, r * lda).reshape(r, lda)[:, :n] @ _arr(x, n)
        elif name == "psc_block_combine":
            y, base, f, mix, A, lda, r, c = a[:8]
            v = _arr(base, n).copy()
            if f.value:
                v += mix * _arr(f, n)
            if r:
                v -= _arr(c, r) @ _arr(A, r * lda).reshape(r, lda)[:, :n]
            _arr(y, n)[:] = v
        elif name == "psc_block_absrow_max":
            A, lda, r, out = a[:4]
            _arr(out, 1)[0] = np.abs(_arr(A, r * lda).reshape(r, lda)[:, :n]).sum(axis=0).max()
        elif name == "psc_gram":
            dtype, A, lda, B, ldb, k, mode, out = a[:8]
            assert dtype == F64 and mode == 0
            G = _arr(A, k * lda).reshape(k, lda)[:, :n] @ _arr(B, k * ldb).reshape(k, ldb)[:, :n].T
            _arr(out, k * k)[:] = G.T.ravel()   # column-major
        elif name == "psc_gemm_nn":
            dtype, W, ldw, k, Q, kout, out, ldo = a[:8]
            Wm = _arr(W, k * ldw).reshape(k, ldw)[:, :n]          # rows = the block's columns
            Qm = _arr(Q, k * kout).reshape(kout, k).T             # column-major k x kout
            _arr(out, kout * ldo).reshape(kout, ldo)[:, :n] = (Wm.T @ Qm).T
        else:
            raise AssertionError(f"unexpected entry point {name}")


@pytest.fixture(autouse=True)
def _no_stream(monkeypatch):
    monkeypatch.setattr(gpu, "_stream", lambda: None)


@pytest.mark.parametrize("name,group_size", [("anderson", 0), ("group2", 2)])
def test_mixer2_host_flow_reproduces_reference_outputs(golden_dir, name, group_size):
    """The reference's msecant2 sequences (tests/golden/ref_mixer2.npz): the
    restart at step 9, then the alternating EN stages."""
    g = np.load(golden_dir / "ref_mixer2.npz")
    n = g[f"{name}_x"].shape[1]
    m = gpu.Mixer2(HostContext(n), capacity=20, group_size=group_size)
    for i in range(len(g[f"{name}_x"])):
        out, used = m(torch.from_numpy(g[f"{name}_x"][i].copy()), torch.from_numpy(g[f"{name}_f"][i].copy()))
        assert used == int(g[f"{name}_m"][i]), i
        ref = g[f"{name}_out"][i]
        assert np.abs(out.numpy() - ref).max() <= 1e-11 * np.abs(ref).max(), i


@pytest.mark.parametrize("group_size", [0, 3])
def test_mixer2_host_flow_matches_oracle_over_long_histories(group_size):
    """30 steps of a contracting fixed-point map: histories past 16 columns
    and, with groups of 3, full groups orthogonalised against and the last
    group's DF replaced by DF C."""
    n = 600
    rng = np.random.default_rng(70 + group_size)
    q = np.linalg.qr(rng.standard_normal((n, 16)))[0]
    lam = np.linspace(0.2, 0.97, 16)
    b = rng.standard_normal(n)
    ora = O.MSecant2(group_size=group_size)
    dev = gpu.Mixer2(HostContext(n), capacity=40, group_size=group_size)
    x = rng.standard_normal(n)
    for i in range(30):
        f = b + q @ (lam * (q.T @ x)) + 0.05 * np.tanh(x) - x
        xo, mo = ora(x, f)
        xd, md = dev(torch.from_numpy(x.copy()), torch.from_numpy(f.copy()))
        assert md == mo, i
        assert np.abs(xd.numpy() - xo).max() <= 1e-8 * np.abs(xo).max(), i
        x = xo
