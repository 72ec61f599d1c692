"""pwb200 -- the B200 (sm_100a) hot path of PWDFT.jl behind its own API.

The functions below mirror PWDFT.jl's operator interface for the path
(op_H.jl, op_K.jl, op_V_loc.jl, op_V_Ps_nloc.jl, Kprec.jl, calc_rhoe.jl):
same names (Julia's trailing ``!`` becomes a trailing ``_``), same argument
meaning, same accumulate/overwrite semantics and the same hidden
``Ham.ik`` / ``Ham.ispin`` state.  Every call goes to libpwb200.so through
its C ABI; there is no CPU fallback.

Wavefunctions on the device are torch tensors of shape (Nstates, Ngw)
(row = band), the memory layout of the reference's column-major
Matrix{ComplexF64}(Ngw, Nstates).  complex128 selects the FP64 path,
complex64 the mixed-precision path.
"""
from ._lib import (PWError, PW_C128, PW_C64, PW_OP_K, PW_OP_VLOC, PW_OP_VNL, PW_OP_H, PW_ACCUMULATE, lib,
                   LIB_PATH)
from .context import Context
from .system import Hamiltonian, System, Basis, GTH

__all__ = ["Hamiltonian", "System", "Basis", "GTH", "Context", "PWError", "op_H", "op_H_", "op_K_", "op_V_loc_",
           "op_V_Ps_nloc_", "Kprec", "Kprec_", "calc_rhoe_", "lib", "LIB_PATH"]


def _torch():
    import torch
    return torch


def op_H_(Ham, psi, Hpsi):
    """op_H!(Ham, psi, Hpsi): Hpsi = (K + V_loc + V_Ps_nloc) psi (op_H.jl:53-63)."""
    ops = PW_OP_K | PW_OP_VLOC | (PW_OP_VNL if Ham.NbetaNL > 0 else 0)
    Ham.ctx.apply(Ham.ik, Ham.ispin, psi, Hpsi, ops)


def op_H(Ham, psi):
    """op_H(Ham, psi) -> new array (op_H.jl:4-27)."""
    Hpsi = _torch().empty_like(psi)
    op_H_(Ham, psi, Hpsi)
    return Hpsi


def op_K_(Ham, psi, Hpsi):
    """op_K!(Ham, psi, Hpsi): Hpsi += 0.5|G+k|^2 psi (op_K.jl:44-75)."""
    Ham.ctx.apply(Ham.ik, Ham.ispin, psi, Hpsi, PW_OP_K | PW_ACCUMULATE)


def op_V_loc_(Ham, psi, Hpsi):
    """op_V_loc!(Ham, psi, Hpsi): Hpsi += V_loc psi (op_V_loc.jl:108-167)."""
    Ham.ctx.apply(Ham.ik, Ham.ispin, psi, Hpsi, PW_OP_VLOC | PW_ACCUMULATE)


def op_V_Ps_nloc_(Ham, psi, Hpsi):
    """op_V_Ps_nloc!(Ham, psi, Hpsi): Hpsi += sum h_ij beta_i <beta_j|psi>
    (op_V_Ps_nloc.jl:39-78)."""
    Ham.ctx.apply(Ham.ik, Ham.ispin, psi, Hpsi, PW_OP_VNL | PW_ACCUMULATE)


def Kprec_(ik, Ham, psi, Kpsi):
    """Kprec!(ik, pw, psi, Kpsi) (Kprec.jl:30-44)."""
    Ham.ctx.kprec(ik, psi, Kpsi)


def Kprec(ik, Ham, psi):
    """Kprec(ik, pw, psi) (Kprec.jl:10-28)."""
    out = _torch().empty_like(psi)
    Ham.ctx.kprec(ik, psi, out)
    return out


def calc_rhoe_(Ham, psiks, Rhoe, Focc):
    """calc_rhoe!(Ham, psiks, Rhoe) for Nspin = 1 without symmetrisation
    (calc_rhoe.jl:9-135): Rhoe (torch float64, N) is overwritten.
    Focc: (Nstates, Nkpt) occupations."""
    for ik, psi in enumerate(psiks):
        w = Ham.wk[ik] * Focc[:, ik]
        Ham.ctx.calc_rhoe(ik, psi, w, Rhoe, accumulate=(ik > 0))


# ---- eigensolvers and orthonormalisation under the reference's names ----
# (Nspin = 1: psiks holds one (Nstates, Ngw) device block per k-point; the
# returned evals are (Nstates, Nkpt) like the reference's (Nstates, Nkspin).)

def diag_LOBPCG_(Ham, psiks, tol=1e-5, NiterMax=100, Nstates_conv=0, verbose=False, verbose_last=False):
    """diag_LOBPCG!(Ham, psiks; tol, NiterMax, verbose, verbose_last,
    Nstates_conv) (diag_LOBPCG.jl:1-28): every block replaced by its Ritz
    vectors; returns evals (the print switches are ignored)."""
    import numpy as np
    evals = np.zeros((psiks[0].shape[0], len(psiks)))
    for ik, X in enumerate(psiks):
        Ham.ik = ik
        evals[:, ik], _ = Ham.ctx.lobpcg(ik, Ham.ispin, X, tol=tol, nitermax=NiterMax, nconv=Nstates_conv)
    return evals


def diag_davidson_qe_(Ham, psiks, tol=1e-5, NiterMax=100, verbose=False, verbose_last=False, Nstates_conv=0):
    """diag_davidson_qe!(Ham, psiks; tol, NiterMax, verbose, verbose_last,
    Nstates_conv) (diag_davidson_qe_v2.jl:6-34); like the reference, which
    passes only tol and NiterMax on to the per-k solver, Nstates_conv and the
    print switches have no effect."""
    import numpy as np
    evals = np.zeros((psiks[0].shape[0], len(psiks)))
    for ik, X in enumerate(psiks):
        Ham.ik = ik
        evals[:, ik], _ = Ham.ctx.davidson(ik, Ham.ispin, X, tol=tol, nitermax=NiterMax)
    return evals


def diag_CheFSI_(Ham, psiks, cheby_degree, seed=1234):
    """diag_CheFSI!(Ham, psiks, cheby_degree) (CheFSI.jl:1-31); the Lanczos
    start vectors come from a generator seeded with `seed`."""
    import numpy as np
    from .chefsi import diag_chefsi_k
    rng = np.random.default_rng(seed)
    evals = np.zeros((psiks[0].shape[0], len(psiks)))
    for ik, X in enumerate(psiks):
        Ham.ik = ik
        evals[:, ik] = diag_chefsi_k(Ham.ctx, ik, Ham.ispin, X, cheby_degree, rng)
    return evals


def chebyfilt(Ham, X, degree, lb, ub):
    """chebyfilt(Ham, X, degree, lb, ub) -> Y (CheFSI.jl:34-64) at Ham.ik."""
    Y = _torch().empty_like(X)
    Ham.ctx.chebyfilt(Ham.ik, Ham.ispin, X, Y, degree, lb, ub)
    return Y


def get_ub_lb_lanczos(Ham, nlancz, v0=None, seed=None):
    """get_ub_lb_lanczos(Ham, nlancz) -> (ub, lb) (CheFSI.jl:67-125) at Ham.ik;
    v0 (complex128 device vector of Ngw) defaults to a seeded normal draw,
    where the reference calls randn."""
    import numpy as np
    if v0 is None:
        ngw = Ham.ctx.Ngw[Ham.ik]
        rng = np.random.default_rng(seed)
        v0 = _torch().from_numpy(rng.standard_normal(ngw) + 1j * rng.standard_normal(ngw)).to(f"cuda:{Ham.ctx.device}")
    return Ham.ctx.lanczos_bounds(Ham.ik, Ham.ispin, nlancz, v0)


def ortho_sqrt_(Ham, psi):
    """ortho_sqrt!(psi) (ortho_sqrt.jl:1-11), in place on the device (the
    context of Ham runs it)."""
    Ham.ctx.ortho_sqrt(psi)


__all__ += ["diag_LOBPCG_", "diag_davidson_qe_", "diag_CheFSI_", "chebyfilt", "get_ub_lb_lanczos", "ortho_sqrt_"]


def diag_davidson_(Ham, psiks, tol=1e-5, NiterMax=100, Nstates_conv=0, verbose=False, verbose_last=False):
    """diag_davidson!(Ham, psiks; tol, NiterMax, verbose, verbose_last,
    Nstates_conv) (diag_davidson.jl:12-38): the 2-block Davidson per k-point
    on complex128 blocks (pwb200.davidson; the print switches are ignored)."""
    import numpy as np
    from .davidson import diag_davidson_k
    evals = np.zeros((psiks[0].shape[0], len(psiks)))
    for ik, X in enumerate(psiks):
        Ham.ik = ik
        evals[:, ik], _ = diag_davidson_k(Ham.ctx, ik, Ham.ispin, X, tol=tol, NiterMax=NiterMax,
                                          Nstates_conv=Nstates_conv)
    return evals


__all__ += ["diag_davidson_"]


# The reference's keyword names that are not ASCII, and its print switches
# (output only, accepted and ignored)
_KW_RENAME = {"\u03b1_t": "alpha_t", "\u03b1_max": "alpha_max"}
_KW_PRINT = ("verbose_last", "print_final_ebands", "print_final_energies")


def _reference_kwargs(kwargs):
    out = {}
    for k, v in kwargs.items():
        if k in _KW_PRINT:
            continue
        out[_KW_RENAME.get(k, k)] = v
    return out


def diag_Emin_PCG_(Ham, psiks, tol=1e-5, NiterMax=100, Nstates_conv=0, tol_ebands=1e-4, alpha_t=3e-5, I_CG_BETA=2,
                   verbose=False, **kwargs):
    """diag_Emin_PCG!(Ham, psiks; tol, NiterMax, Nstates_conv, tol_ebands, α_t, I_CG_BETA)
    (diag_Emin_PCG.jl:17-47): all-band PCG per k-point on complex128 blocks
    (pwb200.emin_pcg).  The reference's own keyword names (α_t, verbose,
    verbose_last) are accepted as well."""
    import numpy as np
    from .emin_pcg import diag_Emin_PCG_k
    kw = _reference_kwargs(kwargs)
    alpha_t = kw.pop("alpha_t", alpha_t)
    if kw:
        raise TypeError("diag_Emin_PCG_: unexpected keyword arguments %s" % sorted(kw))
    evals = np.zeros((psiks[0].shape[0], len(psiks)))
    for ik, X in enumerate(psiks):
        Ham.ik = ik
        evals[:, ik], _ = diag_Emin_PCG_k(Ham.ctx, ik, Ham.ispin, X, tol=tol, NiterMax=NiterMax,
                                          Nstates_conv=Nstates_conv, tol_ebands=tol_ebands, alpha_t=alpha_t,
                                          I_CG_BETA=I_CG_BETA)
    return evals


__all__ += ["diag_Emin_PCG_"]


def KS_solve_SCF_(Ham, **kwargs):
    """KS_solve_SCF!(Ham; ...) (KS_solve_SCF.jl:24-373): pwb200.scf.KS_solve_SCF
    (update_psi "LOBPCG" | "davidson" | "CheFSI" | "PCG", precision "fp64" |
    "mixed", smearing, symmetry, k-point sharding over a process group).  The
    reference's print switches are accepted and ignored."""
    from .scf import KS_solve_SCF
    return KS_solve_SCF(Ham, **_reference_kwargs(kwargs))


def KS_solve_Emin_PCG_(Ham, psiks=None, **kwargs):
    """KS_solve_Emin_PCG!(Ham, psiks; ...) (KS_solve_Emin_PCG.jl:27-270):
    pwb200.emin_scf.KS_solve_Emin_PCG.  The reference's keyword names α_t and
    α_max are accepted for alpha_t and alpha_max, its print switches are
    ignored."""
    from .emin_scf import KS_solve_Emin_PCG
    return KS_solve_Emin_PCG(Ham, psiks, **_reference_kwargs(kwargs))


__all__ += ["KS_solve_SCF_", "KS_solve_Emin_PCG_"]
