"""The 2-block diag_davidson! (diag_davidson.jl:50-191) on the device, one
k-point at a time, assembled from the library's block operations:

  H X, H R                  pw_apply
  R <- Kprec(R)             pw_kprec
  X'HX, X'HR, R'HR, X'R, R'R and the residual norms    pw_gram (FP64 output)
  X diag(e) - HX, R diag(1/|r|), [X R] Xred, [HX HR] Xred     pw_rotate
  eigen(Hermitian(Hred), Hermitian(Sred)), lowest Nstates      pw_eigh

The 2 Nstates x 2 Nstates reduced matrices are assembled on the host, as in
the reference.  FP64 blocks only: the basis [X, R] is not orthogonalised, so
its overlap Sred loses definiteness in FP32 as the residuals shrink, and the
reference has no other precision.
"""
import numpy as np

EPS = np.finfo(np.float64).eps


def _gram_host(ctx, A, B):
    """A^H B (host complex128, m x n) for band-major device blocks A, B."""
    import torch
    out = torch.zeros((B.shape[0], A.shape[0]), dtype=torch.complex128, device=A.device)
    ctx.gram(A, B, out)
    return out.cpu().numpy().T


def _rotate(ctx, A, U, out, accumulate=False):
    """out (+)= A U for a band-major device block A and a host k x n matrix U."""
    import torch
    Ud = torch.from_numpy(np.ascontiguousarray(np.asarray(U, dtype=np.complex128).T)).to(A.device)
    ctx.rotate(A, Ud, out, accumulate=accumulate)


def _residual(ctx, X, HX, evals):
    """R = X diag(evals) - HX and |R_i| (diag_davidson.jl:88-93, :157-162)."""
    import torch
    R = torch.neg(HX)
    _rotate(ctx, X, np.diag(evals), R, accumulate=True)
    res = np.sqrt(np.maximum(np.real(np.diag(_gram_host(ctx, R, R))), 0.0))
    return R, res


def diag_davidson_k(ctx, ik, ispin, X, tol=1e-5, NiterMax=100, Nstates_conv=0):
    """diag_davidson!(Ham, X; tol, NiterMax, Nstates_conv) for k-point ik: X
    (torch complex128 (Nstates, Ngw) device block, orthonormal on entry) is
    overwritten with the Ritz vectors.  Returns (evals, iterations)."""
    import torch
    if X.dtype != torch.complex128:
        raise TypeError("diag_davidson! runs on complex128 blocks (the reference's FP64 path)")
    n = X.shape[0]
    if Nstates_conv == 0:
        Nstates_conv = n
    s1, s2 = slice(0, n), slice(n, 2 * n)
    HX = torch.empty_like(X)
    ctx.apply(ik, ispin, X, HX)
    evals = np.real(np.diag(_gram_host(ctx, X, HX)))                    # :82-85
    R, res = _residual(ctx, X, HX, evals)
    evals_old = evals.copy()
    Hred = np.zeros((2 * n, 2 * n), dtype=np.complex128)
    Sred = np.zeros_like(Hred)
    it = 0
    for it in range(1, NiterMax + 1):
        res_norm = np.where(EPS < res, 1.0 / np.where(res > 0, res, 1.0), 1.0)   # :107-117
        Rs = torch.zeros_like(R)
        _rotate(ctx, R, np.diag(res_norm), Rs)
        R = torch.empty_like(Rs)
        ctx.kprec(ik, Rs, R)                                            # :119
        HR = torch.empty_like(R)
        ctx.apply(ik, ispin, R, HR)                                     # :121
        Hred[s1, s1] = _gram_host(ctx, X, HX) if it == 1 else np.diag(evals.astype(np.complex128))
        Hred[s1, s2] = _gram_host(ctx, X, HR)                           # :133-136
        Hred[s2, s2] = _gram_host(ctx, R, HR)
        Hred[s2, s1] = Hred[s1, s2].conj().T
        Sred[s1, s1] = np.eye(n)                                        # :138-141
        Sred[s1, s2] = _gram_host(ctx, X, R)
        Sred[s2, s2] = _gram_host(ctx, R, R)
        Sred[s2, s1] = Sred[s1, s2].conj().T
        Hred = 0.5 * (Hred + Hred.conj().T)                             # :143-144
        Sred = 0.5 * (Sred + Sred.conj().T)
        T = torch.from_numpy(np.ascontiguousarray(Hred.T)).to(X.device)
        G = torch.from_numpy(np.ascontiguousarray(Sred.T)).to(X.device)
        lam, S = ctx.eigh(T, G, k=n)                                    # :146
        evals = lam.cpu().numpy().copy()
        Xr = S.cpu().numpy().T                                          # 2n x n
        nconv = int(np.sum(np.abs(evals - evals_old) < tol))            # :150-151
        Xn = torch.zeros_like(X)                                        # :153-154
        _rotate(ctx, X, Xr[s1, :], Xn)
        _rotate(ctx, R, Xr[s2, :], Xn, accumulate=True)
        HXn = torch.zeros_like(HX)
        _rotate(ctx, HX, Xr[s1, :], HXn)
        _rotate(ctx, HR, Xr[s2, :], HXn, accumulate=True)
        X.copy_(Xn)
        HX = HXn
        R, res = _residual(ctx, X, HX, evals)                           # :157-162
        if nconv >= Nstates_conv:                                       # :170-176
            break
        evals_old = evals.copy()
    return evals, it
