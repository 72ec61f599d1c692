"""The 2-block diag_davidson! (diag_davidson.jl:50-191).

CPU: the oracle restatement converges to the exact lowest eigenvalues of
Si fcc's dense H(Gamma); the device composition (pwb200.davidson) run on a
NumPy stand-in for the library's block operations, whose layouts follow the
C ABI (pw_gram writes A^H B column-major, pw_rotate takes U column-major,
pw_eigh returns eigenvectors as rows), reproduces the oracle's iterations
and eigenvalues.
GPU: the same composition on the real library against the exact spectrum
(FP64, 1e-9 Ha at tol 1e-10).
"""
import numpy as np
import pytest
import scipy.linalg as sla

from conftest import cuda_ok
from numpy_ctx import NumpyCtx


@pytest.fixture(scope="module")
def fcc_gamma():
    from oracle import systems, ops
    H = systems.Ham_Si_fcc(meshk=(1, 1, 1), extra_states=4)
    H.V_Total = H.V_Ps_loc.copy()          # op_V_loc with the local pseudopotential
    ngw = H.pw.gvecw.Ngw[0]
    Hd = ops.op_H(H, np.eye(ngw, dtype=np.complex128), 0)
    lam = np.linalg.eigvalsh(0.5 * (Hd + Hd.conj().T))
    rng = np.random.default_rng(1)
    X0 = np.linalg.qr(rng.standard_normal((ngw, 8)) + 1j * rng.standard_normal((ngw, 8)))[0]
    return H, lam, X0


def test_oracle_converges(fcc_gamma):
    from oracle import davidson
    H, lam, X0 = fcc_gamma
    X = X0.copy()
    ev, it, conv = davidson.diag_davidson(H, X, 0, tol=1e-10, NiterMax=300)
    assert conv and np.abs(ev - lam[:8]).max() < 1e-8
    assert np.abs(X.conj().T @ X - np.eye(8)).max() < 1e-8


def test_composition_matches_oracle(fcc_gamma):
    import torch
    from oracle import davidson
    from pwb200.davidson import diag_davidson_k
    H, lam, X0 = fcc_gamma
    Xo = X0.copy()
    ev_o, it_o, _ = davidson.diag_davidson(H, Xo, 0, tol=1e-8, NiterMax=200)
    Xd = torch.from_numpy(np.ascontiguousarray(X0.T))
    ev_d, it_d = diag_davidson_k(NumpyCtx(H), 0, 0, Xd, tol=1e-8, NiterMax=200)
    assert abs(it_d - it_o) <= 1
    assert np.abs(ev_d - ev_o).max() < 1e-9
    assert np.abs(ev_d - lam[:8]).max() < 1e-6


@pytest.mark.gpu
def test_davidson2_gpu_exact_spectrum(fcc_gamma):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    import pwb200
    from pwb200.davidson import diag_davidson_k
    H, lam, X0 = fcc_gamma
    pw = H.pw
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(0)])
    try:
        ctx.set_vloc(H.V_Total)
        ctx.set_nonlocal(0, H.betaNL[0])
        ctx.set_nonlocal_coef(H.nl_triplets)
        X = torch.from_numpy(np.ascontiguousarray(X0.T)).cuda()
        ev, it = diag_davidson_k(ctx, 0, 0, X, tol=1e-10, NiterMax=300)
        assert it < 300 and np.abs(ev - lam[:8]).max() < 1e-9
        G = torch.zeros((8, 8), dtype=torch.complex128, device="cuda")
        ctx.gram(X, X, G)
        assert np.abs(G.cpu().numpy() - np.eye(8)).max() < 1e-8
    finally:
        ctx.close()
