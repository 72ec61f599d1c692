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
    """Kprec!(ik, pw, psi, Kpsi) (Kprec.jl:97-111)."""
    Ham.ctx.kprec(ik, psi, Kpsi)


def Kprec(ik, Ham, psi):
    """Kprec(ik, pw, psi) (Kprec.jl:77-95)."""
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
