"""diag_CheFSI! (CheFSI.jl:1-31) on the device, one k-point at a time.

  get_ub_lb_lanczos        pw_lanczos_bounds (nlancz = 2 Nstates, FP64; the start
                           vector, randn in the reference, drawn here from a seeded
                           generator on the host)
  chebyfilt                pw_chebyfilt (degree op_H applications)
  ortho_sqrt!              pw_ortho_sqrt
  Hr = psi' op_H(psi)      pw_apply + pw_gram
  eigvals(Hermitian(Hr))   pw_eigh, eigenvalues only

As in the reference, psi is left as the orthonormalised filtered block (no
rotation to Ritz vectors) and the eigenvalues are those of its Rayleigh
quotient; the density it gives is only rotation-invariant when every state
of the block has the same occupation, which is the reference's behaviour
too.
"""
import numpy as np


def diag_chefsi_k(ctx, ik, ispin, psi, cheby_degree, rng):
    """One k-point of diag_CheFSI!: psi (torch (Nstates, Ngw) device block,
    complex128 or complex64) is replaced in place; returns the Nstates
    eigenvalues of psi' H psi (host, ascending)."""
    import torch
    nb, ngw = psi.shape
    dev = psi.device
    v0 = torch.from_numpy(rng.standard_normal(ngw) + 1j * rng.standard_normal(ngw)).to(dev)
    ub, lb = ctx.lanczos_bounds(ik, ispin, 2 * nb, v0)
    Y = torch.empty_like(psi)
    ctx.chebyfilt(ik, ispin, psi, Y, cheby_degree, lb, ub)
    ctx.ortho_sqrt(Y)
    psi.copy_(Y)
    HY = Y
    ctx.apply(ik, ispin, psi, HY)
    Hr = torch.zeros((nb, nb), dtype=torch.complex128, device=dev)
    ctx.gram(psi, HY, Hr)
    lam, _ = ctx.eigh(Hr, None, k=nb, vectors=False)
    return lam.cpu().numpy()


def diag_CheFSI(ctx, psiks, cheby_degree, iks=None, ispin=0, seed=1234):
    """diag_CheFSI!(Ham, psiks, cheby_degree) over the k-points iks (all by
    default); returns evals (Nstates x len(iks))."""
    rng = np.random.default_rng(seed)
    iks = range(len(psiks)) if iks is None else iks
    return np.stack([diag_chefsi_k(ctx, ik, ispin, psiks[ik], cheby_degree, rng) for ik in iks], axis=1)
