"""The device eigensolvers against SciPy and the FP64 oracle.

  pw_eigh    eigen(T, G) / eigvals(XHX) of diag_LOBPCG.jl:86,185,216
             (LAPACK zhegv/zheev in the reference) vs scipy.linalg.eigh
  pw_lobpcg  diag_LOBPCG! (diag_LOBPCG.jl:51-225) vs the exact spectrum of
             the oracle's dense Hamiltonian and vs the oracle's own LOBPCG
  pw_davidson diag_davidson_qe! (diag_davidson_qe_v2.jl:38-216) likewise
Tolerances: FP64 eigenvalues 1e-9 Ha (tol 1e-10), mixed 5e-5 Ha (tol 1e-5,
the SCF's floor ethr_evals_last, KS_solve_SCF.jl:42).
"""
import numpy as np
import pytest
import scipy.linalg as sla

from conftest import cuda_ok

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx_fcc():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import pwb200
    from oracle import systems
    H = systems.Ham_Si_fcc(meshk=(2, 2, 2), extra_states=4)
    rng = np.random.default_rng(3)
    H.V_Total = H.V_Ps_loc + 0.05 * np.cos(np.arange(H.pw.Npoints) * 0.37)
    pw = H.pw
    ctx = pwb200.Context(pw.Ns, pw.CellVolume, pw.gvecw.idx_gw2r, [pw.Gk2(k) for k in range(pw.kpoints.Nkpt)])
    ctx.set_vloc(H.V_Total)
    for ik in range(pw.kpoints.Nkpt):
        ctx.set_nonlocal(ik, H.betaNL[ik])
    ctx.set_nonlocal_coef(H.nl_triplets)
    yield H, ctx, rng
    ctx.close()


def dev_colmajor(A):
    """A column-major n x n matrix as a torch (n, n) tensor (its transpose)."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(A.T)).cuda()


@pytest.mark.parametrize("n,k", [(40, 40), (150, 50), (333, 111)])
def test_eigh_generalized(ctx_fcc, n, k):
    H, ctx, rng = ctx_fcc
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    ev = np.sort(rng.standard_normal(n))
    ev[3:6] = ev[3]            # a 3-fold and a 2-fold degeneracy
    ev[10:12] = ev[10]
    T = (Q * ev) @ Q.conj().T
    B = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    G = B @ B.conj().T / n + np.eye(n)
    ref = sla.eigh(T, G, eigvals_only=True)[:k]
    Tt, Gt = dev_colmajor(np.triu(T)), dev_colmajor(np.triu(G))   # only the upper triangles are read
    lam, S = ctx.eigh(Tt, Gt, k=k)
    lam = lam.cpu().numpy()
    S = S.cpu().numpy().T            # n x k
    scale = np.abs(ev).max()
    assert np.abs(lam - ref).max() < 1e-11 * scale
    assert np.abs(T @ S - G @ S * lam).max() < 1e-10 * scale
    assert np.abs(S.conj().T @ G @ S - np.eye(k)).max() < 1e-10


def test_eigh_standard_and_errors(ctx_fcc):
    import torch
    import pwb200
    H, ctx, rng = ctx_fcc
    n = 64
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    A = A + A.conj().T
    lam, _ = ctx.eigh(dev_colmajor(A), None, k=n, vectors=False)
    assert np.abs(lam.cpu().numpy() - np.linalg.eigvalsh(A)).max() < 1e-11 * np.abs(A).max()
    Gbad = -np.eye(n, dtype=np.complex128)
    with pytest.raises(pwb200.PWError) as e:
        ctx.eigh(dev_colmajor(A), dev_colmajor(Gbad), k=4)
    assert e.value.status == pwb200._lib.PW_ERR_NOT_POSDEF
    ctx.check_device()


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_lobpcg_matches_exact_spectrum(ctx_fcc, prec):
    import torch
    from oracle import ops, lobpcg
    H, ctx, rng = ctx_fcc
    ik = 1
    ngw = H.pw.gvecw.Ngw[ik]
    nb = 8
    Hd = ops.op_H(H, np.eye(ngw, dtype=np.complex128), ik)       # dense H(k)
    exact = np.linalg.eigvalsh(0.5 * (Hd + Hd.conj().T))[:nb]
    X0 = lobpcg.ortho_sqrt(rng.standard_normal((ngw, nb)) + 1j * rng.standard_normal((ngw, nb)))
    dt = torch.complex128 if prec == "c128" else torch.complex64
    X = torch.from_numpy(np.ascontiguousarray(X0.T)).cuda().to(dt).contiguous()
    tol = 1e-10 if prec == "c128" else 1e-5
    ev, nit = ctx.lobpcg(ik, 0, X, tol=tol, nitermax=300)
    bound = 1e-9 if prec == "c128" else 5e-5
    assert np.abs(ev - exact).max() < bound, (ev - exact, nit)
    # the oracle's LOBPCG from the same start converges to the same values
    # (two independently converged runs: each is within its own tolerance)
    Xo = X0.copy()
    evo = lobpcg.diag_LOBPCG_k(H, Xo, ik, tol=tol, NiterMax=300)
    assert np.abs(ev - evo).max() < (1e-9 if prec == "c128" else 2e-4)
    # returned vectors are orthonormal Ritz vectors; in the mixed path the
    # split-BF16x3 products carry ~2^-17 relative error per term, so the
    # Gram matrices that orthonormalise X are good to a few 1e-5
    Xr = X.cpu().numpy().T.astype(np.complex128)
    assert np.abs(Xr.conj().T @ Xr - np.eye(nb)).max() < (1e-10 if prec == "c128" else 5e-5)


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_ortho_sqrt(ctx_fcc, prec):
    """ortho_sqrt (ortho_sqrt.jl:1-4) against the oracle's."""
    import torch
    from oracle import lobpcg
    H, ctx, rng = ctx_fcc
    ngw = H.pw.gvecw.Ngw[0]
    psi = rng.random((ngw, 12)) + 1j * rng.random((ngw, 12))
    ref = lobpcg.ortho_sqrt(psi)
    dt = torch.complex128 if prec == "c128" else torch.complex64
    X = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda().to(dt).contiguous()
    ctx.ortho_sqrt(X)
    got = X.cpu().numpy().T.astype(np.complex128)
    assert np.abs(got - ref).max() < (1e-10 if prec == "c128" else 5e-4)
    assert np.abs(got.conj().T @ got - np.eye(12)).max() < (1e-12 if prec == "c128" else 1e-4)


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_ortho_cholesky(ctx_fcc, prec):
    """ortho_cholesky! (ortho_sqrt.jl:80-89) against the oracle."""
    import torch
    from oracle import lobpcg
    H, ctx, rng = ctx_fcc
    ngw = H.pw.gvecw.Ngw[0]
    psi = rng.standard_normal((ngw, 8)) + 1j * rng.standard_normal((ngw, 8))
    ref = lobpcg.ortho_cholesky(psi)
    dt = torch.complex128 if prec == "c128" else torch.complex64
    X = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda().to(dt).contiguous()
    ctx.ortho_cholesky(X)
    got = X.cpu().numpy().T.astype(np.complex128)
    tol = 1e-11 if prec == "c128" else 2e-5
    assert np.abs(got - ref).max() < tol * np.abs(ref).max()
    assert np.abs(got.conj().T @ got - np.eye(8)).max() < (1e-11 if prec == "c128" else 5e-5)


@pytest.mark.parametrize("prec", ["c128", "c64"])
@pytest.mark.parametrize("frac", [False, True])
def test_calc_grad(ctx_fcc, prec, frac):
    """calc_grad (calc_grad.jl:1-57) against the oracle, integer occupations
    and fractional ones (the psi (Hred F - F Hred)/2 term)."""
    import torch
    from oracle import ops, lobpcg
    H, ctx, rng = ctx_fcc
    ik = 1
    ngw = H.pw.gvecw.Ngw[ik]
    psi = lobpcg.ortho_sqrt(rng.standard_normal((ngw, 8)) + 1j * rng.standard_normal((ngw, 8)))
    Focc = np.linspace(2.0, 0.3, 8) if frac else np.full(8, 2.0)
    wk = float(H.pw.kpoints.wk[ik])
    ref = ops.calc_grad(H, psi, ik, Focc, wk)
    dt = torch.complex128 if prec == "c128" else torch.complex64
    X = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda().to(dt).contiguous()
    g = ctx.calc_grad(ik, 0, X, Focc, wk)
    got = g.cpu().numpy().T.astype(np.complex128)
    # mixed: the FP32 op_H (2e-5) plus the split-BF16x3 rotation psi Hred,
    # whose terms (|Hred| ~ 10 Ha for random vectors) cancel against H psi
    tol = 1e-11 if prec == "c128" else 1e-4
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < tol, err


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_davidson_matches_exact_spectrum(ctx_fcc, prec):
    """pw_davidson against the exact spectrum and against the oracle's
    Davidson from the same start: the FP64 path takes the same steps (same
    iteration count, restarts included), the mixed one converges to within
    its FP32 floor."""
    import torch
    from oracle import ops, lobpcg, davidson
    H, ctx, rng = ctx_fcc
    ik = 1
    ngw = H.pw.gvecw.Ngw[ik]
    nb = 8
    Hd = ops.op_H(H, np.eye(ngw, dtype=np.complex128), ik)
    exact = np.linalg.eigvalsh(0.5 * (Hd + Hd.conj().T))[:nb]
    X0 = lobpcg.ortho_sqrt(rng.standard_normal((ngw, nb)) + 1j * rng.standard_normal((ngw, nb)))
    dt = torch.complex128 if prec == "c128" else torch.complex64
    X = torch.from_numpy(np.ascontiguousarray(X0.T)).cuda().to(dt).contiguous()
    tol = 1e-10 if prec == "c128" else 1e-5
    ev, nit = ctx.davidson(ik, 0, X, tol=tol, nitermax=100)
    bound = 1e-9 if prec == "c128" else 5e-5
    assert np.abs(ev - exact).max() < bound, (ev - exact, nit)
    Xo = X0.copy()
    evo, nito = davidson.diag_davidson_qe(H, Xo, ik, EBANDS_THR=tol, NiterMax=100)
    assert np.abs(ev - evo).max() < (1e-9 if prec == "c128" else 2e-4)
    Xr = X.cpu().numpy().T.astype(np.complex128)
    assert np.abs(Xr.conj().T @ Xr - np.eye(nb)).max() < (1e-10 if prec == "c128" else 5e-5)
    if prec == "c128":
        assert nit == nito, (nit, nito)
        # Ritz vectors agree up to a phase per column
        ph = np.sum(Xo.conj() * Xr, axis=0)
        assert np.abs(np.abs(ph) - 1).max() < 1e-8


def test_davidson_iterates_match_oracle(ctx_fcc):
    """A fixed number of FP64 Davidson iterations (NiterMax = 3, so the last
    one returns unconverged) gives the oracle's Ritz values and vectors:
    the device follows the reference step by step, restart included (nb = 4,
    Nvecx = 8, so the basis refreshes after the first expansion)."""
    import torch
    from oracle import lobpcg, davidson
    H, ctx, rng = ctx_fcc
    ik = 0
    ngw = H.pw.gvecw.Ngw[ik]
    nb = 4
    X0 = lobpcg.ortho_sqrt(rng.standard_normal((ngw, nb)) + 1j * rng.standard_normal((ngw, nb)))
    X = torch.from_numpy(np.ascontiguousarray(X0.T)).cuda().contiguous()
    ev, nit = ctx.davidson(ik, 0, X, tol=1e-14, nitermax=3)
    Xo = X0.copy()
    evo, nito = davidson.diag_davidson_qe(H, Xo, ik, EBANDS_THR=1e-14, NiterMax=3)
    assert nit == nito == 3
    assert np.abs(ev - evo).max() < 1e-11
    Xr = X.cpu().numpy().T
    ph = np.sum(Xo.conj() * Xr, axis=0)
    assert np.abs(Xr - Xo * (ph / np.abs(ph))[None, :]).max() < 1e-9


@pytest.mark.parametrize("prec", ["c128", "c64"])
def test_davidson_host_dropin(ctx_fcc, prec):
    """pw_davidson_host on the reference's host array (Ngw x nb, column-major).
    nb = 7: at this k-point the 6th and 7th levels are 5e-5 Ha apart, which a
    6-vector Davidson resolves only slowly (the oracle takes > 100 steps)."""
    import pwb200
    from oracle import ops, lobpcg
    H, ctx, _ = ctx_fcc
    rng = np.random.default_rng(11)
    ik = 2
    ngw = H.pw.gvecw.Ngw[ik]
    Hd = ops.op_H(H, np.eye(ngw, dtype=np.complex128), ik)
    exact = np.linalg.eigvalsh(0.5 * (Hd + Hd.conj().T))[:7]
    evc = np.asfortranarray(lobpcg.ortho_sqrt(rng.standard_normal((ngw, 7)) + 1j * rng.standard_normal((ngw, 7))))
    code = pwb200.PW_C128 if prec == "c128" else pwb200.PW_C64
    ev, nit = ctx.davidson_host(ik, 0, evc, tol=1e-10 if prec == "c128" else 1e-5, nitermax=100, dtype=code)
    assert np.abs(ev - exact).max() < (1e-9 if prec == "c128" else 5e-5), (ev - exact, nit)
    assert np.abs(evc.conj().T @ evc - np.eye(7)).max() < (1e-10 if prec == "c128" else 5e-5)
