"""Chebyshev-filtered subspace iteration.

Oracle (test infrastructure only).  Restates PWDFT.jl CheFSI.jl:
  diag_CheFSI!          :1-31    per k-point: Lanczos bounds, filter,
                                 ortho_sqrt!, eigvals of psi' H psi
  chebyfilt             :36-67   three-term recurrence, sigma1 fixed
  get_ub_lb_lanczos     :70-123  Lanczos with one step of full
                                 reorthogonalisation; lb = eigvals(T)[nlancz/2],
                                 ub = norm_matrix_induced(T) + norm(f)
  norm_matrix_induced   :127-137 ||A 1/sqrt(N)||
The reference draws the Lanczos start vector with randn; here it is an
argument (v0), so the restatement is deterministic.  eigvals(T) of the
non-symmetric Lanczos matrix is taken with numpy's general eigvals, sorted
by real part as Julia sorts real spectra.
"""
import numpy as np
import scipy.linalg as sla

from .ops import op_H
from .lobpcg import ortho_sqrt


def chebyfilt(Ham, X, degree, lb, ub, ik=None):
    """CheFSI.jl:34-64."""
    ik = Ham.ik if ik is None else ik
    ee = (ub - lb) / 2
    c = (ub + lb) / 2
    sigma = ee / (lb - ub)
    sigma1 = sigma
    Y = op_H(Ham, X, ik) - X * c
    Y = Y * sigma1 / ee
    for _ in range(2, degree + 1):
        sigma2 = 1 / (2 / sigma1 - sigma)
        Y1 = (op_H(Ham, Y, ik) - Y * c) * 2 * sigma2 / ee - X * (sigma * sigma2)
        X = Y
        Y = Y1
        sigma = sigma2
    return Y


def norm_matrix_induced(A):
    """CheFSI.jl:128-138."""
    N = A.shape[0]
    v1 = np.ones(N) / np.sqrt(N)
    return float(np.linalg.norm(A @ v1))


def get_ub_lb_lanczos(Ham, nlancz, v0, ik=None):
    """CheFSI.jl:67-125 from the start vector v0; returns (ub, lb, T)."""
    ik = Ham.ik if ik is None else ik
    ngw = v0.shape[0]
    V = np.zeros((ngw, nlancz), dtype=np.complex128)
    HV = np.zeros((ngw, nlancz), dtype=np.complex128)
    T = np.zeros((nlancz, nlancz))
    h = np.zeros(nlancz, dtype=np.complex128)
    s = np.zeros(nlancz, dtype=np.complex128)
    V[:, 0] = v0 / np.linalg.norm(v0)
    HV[:, 0] = op_H(Ham, V[:, :1], ik)[:, 0]
    h[0] = np.real(np.vdot(V[:, 0], HV[:, 0]))
    T[0, 0] = h[0].real
    f = HV[:, 0] - V[:, 0] * h[0]
    s[0] = np.vdot(V[:, 0], f)
    h[0] = h[0] + s[0]
    f = f - V[:, 0] * s[0]
    for j in range(1, nlancz):
        beta = np.linalg.norm(f)
        T[j, j - 1] = beta
        V[:, j] = f / beta
        HV[:, j] = op_H(Ham, V[:, j:j + 1], ik)[:, 0]
        for jj in range(j + 1):
            h[jj] = np.vdot(V[:, jj], HV[:, j])
        f = HV[:, j] - V[:, :j + 1] @ h[:j + 1]
        for jj in range(j + 1):
            s[jj] = np.vdot(V[:, jj], f)
            h[jj] = h[jj] + s[jj]
        f = f - V[:, :j + 1] @ s[:j + 1]
        T[:j + 1, j] = np.real(h[:j + 1])
    ev = np.linalg.eigvals(T)
    ev = np.sort(np.real(ev))
    lb = float(ev[nlancz // 2 - 1])
    ub = norm_matrix_induced(T) + float(np.linalg.norm(f))
    return ub, lb, T


def diag_CheFSI_k(Ham, psi, cheby_degree, v0, ik=None):
    """CheFSI.jl:13-27 for one k-point; returns (psi_new, evals)."""
    ik = Ham.ik if ik is None else ik
    Nstates = psi.shape[1]
    ub, lb, _ = get_ub_lb_lanczos(Ham, 2 * Nstates, v0, ik)
    psi = ortho_sqrt(chebyfilt(Ham, psi, cheby_degree, lb, ub, ik))
    Hr = psi.conj().T @ op_H(Ham, psi, ik)
    return psi, sla.eigvalsh(Hr, lower=False)
