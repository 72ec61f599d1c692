"""diag_Emin_PCG! (diag_Emin_PCG.jl:57-193) on the device, one k-point at a
time, assembled from the library's block operations:

  calc_grad_evals (calc_grad.jl:60-82)    pw_calc_grad with every f_i = 1, w_k = 1
  Kprec                                   pw_kprec
  real(sum(conj(a) .* b))                 the real trace of pw_gram(a, b) (FP64)
  ortho_sqrt                              pw_ortho_sqrt
  psi' H psi, its eigenpairs, X evecs     pw_apply + pw_gram, pw_eigh, pw_rotate

The conjugate directions d = -Kg + beta d_old and the trial points X + a d
are elementwise tensor updates; the scalars alpha and beta are host FP64.
FP64 blocks only (the reference's precision).
"""
import numpy as np


def _rtrace(ctx, A, B):
    """real(sum(conj(A) .* B)) = Re tr(A^H B)."""
    import torch
    out = torch.zeros((B.shape[0], A.shape[0]), dtype=torch.complex128, device=A.device)
    ctx.gram(A, B, out)
    return float(torch.real(torch.trace(out)).item())


def _grad(ctx, ik, ispin, X):
    return ctx.calc_grad(ik, ispin, X, np.ones(X.shape[0]), 1.0)


def _ortho(ctx, Y):
    ctx.ortho_sqrt(Y)
    return Y


def _rayleigh(ctx, ik, ispin, X, vectors):
    import torch
    n = X.shape[0]
    HX = torch.empty_like(X)
    ctx.apply(ik, ispin, X, HX)
    Hr = torch.zeros((n, n), dtype=torch.complex128, device=X.device)
    ctx.gram(X, HX, Hr)
    lam, S = ctx.eigh(Hr, None, k=n, vectors=vectors)
    return lam.cpu().numpy().copy(), S


def diag_Emin_PCG_k(ctx, ik, ispin, X, tol=1e-5, NiterMax=100, Nstates_conv=0, tol_ebands=1e-4, alpha_t=3e-5,
                    I_CG_BETA=2):
    """diag_Emin_PCG!(Ham, X; ...) for k-point ik: X (torch complex128
    (Nstates, Ngw) device block, orthonormal on entry) is overwritten with
    the Ritz vectors.  Returns (evals, iterations)."""
    import torch
    if X.dtype != torch.complex128:
        raise TypeError("diag_Emin_PCG! runs on complex128 blocks (the reference's FP64 path)")
    n = X.shape[0]
    if Nstates_conv == 0:
        Nstates_conv = n
    d_old = torch.zeros_like(X)
    g_old = torch.zeros_like(X)
    Kg_old = torch.zeros_like(X)
    beta = 0.0
    Ebands_old = 0.0
    evals_old, _ = _rayleigh(ctx, ik, ispin, X, False)                 # :92-95
    it = 0
    for it in range(1, NiterMax + 1):
        g = _grad(ctx, ik, ispin, X)                                    # :103-104
        Kg = torch.empty_like(g)
        ctx.kprec(ik, g, Kg)
        if it != 1:                                                     # :106-116 (linear in g - g_old)
            if I_CG_BETA == 1:
                beta = _rtrace(ctx, g, Kg) / _rtrace(ctx, g_old, Kg_old)
            elif I_CG_BETA == 2:
                beta = (_rtrace(ctx, g, Kg) - _rtrace(ctx, g_old, Kg)) / _rtrace(ctx, g_old, Kg_old)
            elif I_CG_BETA == 3:
                beta = (_rtrace(ctx, g, Kg) - _rtrace(ctx, g_old, Kg)) / (
                    _rtrace(ctx, g, d_old) - _rtrace(ctx, g_old, d_old))
            else:
                beta = _rtrace(ctx, g, Kg) / (_rtrace(ctx, d_old, g) - _rtrace(ctx, d_old, g_old))
        if beta < 0.0:                                                  # :117-119
            beta = 0.0
        d = torch.add(torch.neg(Kg), d_old, alpha=beta)                 # :121
        Xc = _ortho(ctx, torch.add(X, d, alpha=alpha_t))                # :123-124
        gt = _grad(ctx, ik, ispin, Xc)
        denum = _rtrace(ctx, g, d) - _rtrace(ctx, gt, d)                # :126-131
        alpha = abs(alpha_t * _rtrace(ctx, g, d) / denum) if denum != 0.0 else 0.0
        X.copy_(_ortho(ctx, torch.add(X, d, alpha=alpha)))              # :134
        evals, _ = _rayleigh(ctx, ik, ispin, X, False)                  # :136-139
        Ebands = float(np.sum(evals))
        nconv = int(np.sum(np.abs(evals - evals_old) < tol))
        evals_old = evals.copy()
        if nconv >= Nstates_conv or abs(Ebands - Ebands_old) <= tol_ebands * n:   # :154-167
            break
        g_old, d_old, Kg_old = g, d, Kg                                 # :169-172
        Ebands_old = Ebands
    _ortho(ctx, X)                                                      # :179-184
    lam, S = _rayleigh(ctx, ik, ispin, X, True)
    Xn = torch.zeros_like(X)
    ctx.rotate(X, S, Xn)          # S (n, n): row j = eigenvector j, i.e. the column-major U
    X.copy_(Xn)
    return lam, it
