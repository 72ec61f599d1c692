"""Hamiltonian application, preconditioner and density.

Oracle (test infrastructure only).  Restates PWDFT.jl:
  op_K.jl:44-75              op_K!  (accumulating)
  op_V_loc.jl:108-167        op_V_loc! (collinear, accumulating)
  op_V_Ps_nloc.jl:39-78      op_V_Ps_nloc! for GTH (accumulating)
  PsPotNL.jl:242-254         calc_betaNL_psi
  op_H.jl:53-63              op_H!  (zero, then K + V_loc + V_nloc)
  Kprec.jl:10-28             Kprec
  calc_rhoe.jl:9-135         calc_rhoe! (no symmetrisation, no dual grid)

psi is a (Ngw, Nstates) complex128 array in the reference's column order;
the band loops of the reference are vectorised over bands here, which does
not change the arithmetic of any single band.
"""
import numpy as np

from .ham import G_to_R, R_to_G


def op_K(Ham, psi, Hpsi, ik=None):
    """op_K.jl:44-75: Hpsi += 0.5 |G+k|^2 psi."""
    ik = Ham.ik if ik is None else ik
    Gw2 = Ham.pw.Gk2(ik)
    Hpsi += 0.5 * psi * Gw2[:, None]


def op_V_loc(Ham, psi, Hpsi, ik=None, V=None, chunk=32):
    """op_V_loc.jl:108-167: per band scatter -> G_to_R -> *V -> R_to_G -> gather-add."""
    ik = Ham.ik if ik is None else ik
    pw = Ham.pw
    V = Ham.V_Total if V is None else V
    idx = pw.gvecw.idx_gw2r[ik]
    N = pw.Npoints
    nb = psi.shape[1]
    for b0 in range(0, nb, chunk):
        b1 = min(nb, b0 + chunk)
        ctmp = np.zeros((b1 - b0, N), dtype=np.complex128)
        ctmp[:, idx] = psi[:, b0:b1].T
        ctmp = G_to_R(pw.Ns, ctmp)
        ctmp *= V[None, :]
        ctmp = R_to_G(pw.Ns, ctmp)
        Hpsi[:, b0:b1] += ctmp[:, idx].T


def calc_betaNL_psi(Ham, psi, ik=None):
    """PsPotNL.jl:242-254: betaNL_psi[ist, ibeta] = conj(psi' * betaNL)."""
    ik = Ham.ik if ik is None else ik
    return np.conj(psi.conj().T @ Ham.betaNL[ik])


def op_V_Ps_nloc(Ham, psi, Hpsi, ik=None):
    """op_V_Ps_nloc.jl:39-78: Hpsi += sum h_ij beta_i (beta_j' psi).
    The quintuple rank-1 loop is the product betaNL * D * (betaNL' psi) with
    D the block-diagonal h matrix assembled from the same (ibeta, jbeta)
    pairs (ham.nonlocal_triplets)."""
    ik = Ham.ik if ik is None else ik
    B = calc_betaNL_psi(Ham, psi, ik)            # (Nstates, Nbeta)
    Hpsi += Ham.betaNL[ik] @ (Ham.Dnl @ B.T)


def op_H(Ham, psi, ik=None):
    """op_H.jl:4-27 / 53-63."""
    Hpsi = np.zeros_like(psi)
    op_K(Ham, psi, Hpsi, ik)
    op_V_loc(Ham, psi, Hpsi, ik)
    if Ham.NbetaNL > 0:
        op_V_Ps_nloc(Ham, psi, Hpsi, ik)
    return Hpsi


def Kprec(Ham, psi, ik=None):
    """Kprec.jl:10-28: psi / (1 + |G+k|^2)."""
    ik = Ham.ik if ik is None else ik
    return psi / (1.0 + Ham.pw.Gk2(ik))[:, None]


def calc_rhoe(Ham, psiks, Focc=None, chunk=32):
    """calc_rhoe.jl:9-135 (Nspin = 1, no dual grid); symmetrize_rhoe! at the
    end when the Hamiltonian was built with symmetry (calc_rhoe.jl:129-132)."""
    pw = Ham.pw
    Focc = Ham.Focc if Focc is None else Focc
    N = pw.Npoints
    rho = np.zeros(N)
    scale = N / np.sqrt(pw.CellVolume)
    for ik in range(pw.kpoints.Nkpt):
        psi = psiks[ik]
        idx = pw.gvecw.idx_gw2r[ik]
        nb = psi.shape[1]
        for b0 in range(0, nb, chunk):
            b1 = min(nb, b0 + chunk)
            ctmp = np.zeros((b1 - b0, N), dtype=np.complex128)
            ctmp[:, idx] = psi[:, b0:b1].T
            ctmp = G_to_R(pw.Ns, ctmp) * scale
            w = pw.kpoints.wk[ik] * Focc[b0:b1, ik]
            rho += (w[:, None] * (ctmp.real ** 2 + ctmp.imag ** 2)).sum(axis=0)
    sym = getattr(Ham, "sym", None)
    if sym is not None and sym.Nsyms > 1:
        from .symmetry import symmetrize_rhoe
        rho = symmetrize_rhoe(pw, sym, Ham.symz, rho)
    return rho


def calc_grad(Ham, psi, ik, Focc, wk):
    """calc_grad.jl:1-57: grad_i = wk f_i (H psi_i - sum_j psi_j <psi_j|H psi_i>), plus
    psi (Hred F - F Hred)/2 unless all f are 2 or all are 1."""
    Hpsi = op_H(Ham, psi, ik)
    Hred = psi.conj().T @ Hpsi
    grad = (Hpsi - psi @ Hred) * (wk * Focc)[None, :]
    if not (np.all(Focc == 2.0) or np.all(Focc == 1.0)):
        F = np.diag(Focc)
        grad = grad + psi @ (0.5 * (Hred @ F - F @ Hred))
    return grad
