"""diag_Emin_PCG! (diag_Emin_PCG.jl:57-193).

CPU: the oracle restatement converges to the exact lowest eigenvalues of
Si fcc's dense H(Gamma) for every beta choice; the device composition
(pwb200.emin_pcg) on the NumPy stand-in for the C-ABI block operations
reproduces the oracle's iterations and eigenvalues.
GPU: the same composition on the real library against the exact spectrum
(FP64, 1e-8 Ha).
"""
import numpy as np
import pytest

from conftest import cuda_ok
from numpy_ctx import NumpyCtx


@pytest.fixture(scope="module")
def fcc_gamma():
    from oracle import systems, ops
    H = systems.Ham_Si_fcc(meshk=(1, 1, 1), extra_states=4)
    H.V_Total = H.V_Ps_loc.copy()
    ngw = H.pw.gvecw.Ngw[0]
    Hd = ops.op_H(H, np.eye(ngw, dtype=np.complex128), 0)
    lam = np.linalg.eigvalsh(0.5 * (Hd + Hd.conj().T))
    rng = np.random.default_rng(2)
    X0 = np.linalg.qr(rng.standard_normal((ngw, 8)) + 1j * rng.standard_normal((ngw, 8)))[0]
    return H, lam, X0


@pytest.mark.parametrize("ibeta", [1, 2, 3, 4])
def test_oracle_converges(fcc_gamma, ibeta):
    from oracle import emin_pcg
    H, lam, X0 = fcc_gamma
    X = X0.copy()
    ev, it, conv = emin_pcg.diag_Emin_PCG(H, X, 0, tol=1e-9, NiterMax=400, tol_ebands=1e-12, I_CG_BETA=ibeta)
    assert conv and np.abs(ev - lam[:8]).max() < 1e-7, (ibeta, it)
    assert np.abs(X.conj().T @ X - np.eye(8)).max() < 1e-10


@pytest.mark.parametrize("ibeta", [2, 4])
def test_composition_matches_oracle(fcc_gamma, ibeta):
    import torch
    from oracle import emin_pcg
    from pwb200.emin_pcg import diag_Emin_PCG_k
    H, lam, X0 = fcc_gamma
    Xo = X0.copy()
    ev_o, it_o, _ = emin_pcg.diag_Emin_PCG(H, Xo, 0, tol=1e-9, NiterMax=400, tol_ebands=1e-12, I_CG_BETA=ibeta)
    Xd = torch.from_numpy(np.ascontiguousarray(X0.T))
    ev_d, it_d = diag_Emin_PCG_k(NumpyCtx(H), 0, 0, Xd, tol=1e-9, NiterMax=400, tol_ebands=1e-12, I_CG_BETA=ibeta)
    assert abs(it_d - it_o) <= 1
    assert np.abs(ev_d - ev_o).max() < 1e-9
    # the final rotation leaves the Ritz vectors in X
    Xh = Xd.numpy().T
    from oracle import ops
    R = ops.op_H(H, Xh, 0) - Xh * ev_d[None, :]
    assert np.abs(R).max() < 1e-3


@pytest.mark.gpu
def test_emin_pcg_gpu_exact_spectrum(fcc_gamma):
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    import pwb200
    from pwb200.emin_pcg import diag_Emin_PCG_k
    H, lam, X0 = fcc_gamma
    pw = H.pw
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(0)])
    try:
        ctx.set_vloc(H.V_Total)
        ctx.set_nonlocal(0, H.betaNL[0])
        ctx.set_nonlocal_coef(H.nl_triplets)
        X = torch.from_numpy(np.ascontiguousarray(X0.T)).cuda()
        ev, it = diag_Emin_PCG_k(ctx, 0, 0, X, tol=1e-9, NiterMax=400, tol_ebands=1e-12)
        assert it < 400 and np.abs(ev - lam[:8]).max() < 1e-8
    finally:
        ctx.close()
