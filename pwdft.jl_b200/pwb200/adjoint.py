"""Reverse-mode derivatives of the hot path, as torch.autograd Functions (the
Python analogue of the ChainRulesCore rrules in julia/PWDFTB200.jl).

  local_band_energy(ctx, ik, V, psi, w)
      E = sum_b w_b <psi_b| V_loc |psi_b>  (the op_V_loc part of the band
      energy, op_V_loc.jl:33-92) at fixed psi; its gradient with respect to
      V_loc(r) is pw_vloc_vjp, dE/dV_loc(r) = rho(r) dVol (calc_rhoe.jl:51-78).
  vloc_inner(ctx, ik, V, psi, lam, w)
      L = sum_b w_b Re<lam_b| V_loc psi_b>, gradient pw_vloc_vjp with the
      cotangent lam.
  ionic_energy(Ham, positions, energy, psiks, rho, Focc)
      attaches to a converged total energy its gradient with respect to the
      atomic positions, -F (calc_forces_Ps_loc.jl:13-72,
      calc_forces_Ps_nloc.jl:291-411, calc_forces_NN.jl): pw_forces_local,
      pw_forces_nonlocal and the Ewald forces (Hellmann-Feynman, so psi and
      rho are held fixed).
"""
import numpy as np


def _vjp(ctx, ik, psi, w, lam=None):
    import torch
    dV = torch.zeros(ctx.N, dtype=torch.float64, device=psi.device)
    ctx.vloc_vjp(ik, psi, w, dV, lam=lam)
    return dV


def _functions():
    import torch

    class LocalBandEnergy(torch.autograd.Function):
        @staticmethod
        def forward(fc, ctx, ik, V, psi, w, lam):
            dV = _vjp(ctx, ik, psi, w, lam)
            fc.save_for_backward(dV)
            return torch.dot(V, dV)

        @staticmethod
        def backward(fc, g):
            (dV,) = fc.saved_tensors
            return None, None, g * dV, None, None, None

    class IonicEnergy(torch.autograd.Function):
        @staticmethod
        def forward(fc, positions, energy, F):
            fc.save_for_backward(F)
            return energy.clone()

        @staticmethod
        def backward(fc, g):
            (F,) = fc.saved_tensors
            return -g * F, None, None

    return LocalBandEnergy, IonicEnergy


_FN = None


def _fn():
    global _FN
    if _FN is None:
        _FN = _functions()
    return _FN


def local_band_energy(ctx, ik, V, psi, w):
    """sum_b w_b <psi_b|V|psi_b> for the device potential V (torch float64, N,
    may require grad) and the device block psi (nb, Ngw); differentiable in V."""
    return _fn()[0].apply(ctx, ik, V, psi, np.asarray(w, dtype=np.float64), None)


def vloc_inner(ctx, ik, V, psi, lam, w):
    """sum_b w_b Re<lam_b|V psi_b>, differentiable in V."""
    return _fn()[0].apply(ctx, ik, V, psi, np.asarray(w, dtype=np.float64), lam)


def ionic_energy(Ham, positions, energy, psiks, rho, Focc):
    """The converged total energy as a function of the atomic positions
    (torch (3, natoms) float64, requires grad): backward gives -F from the
    device force kernels and the Ewald term."""
    import torch
    from .forces import calc_forces
    F = torch.from_numpy(np.ascontiguousarray(calc_forces(Ham, psiks, rho, Focc))).to(positions)
    e = torch.as_tensor(float(energy), dtype=torch.float64, device=positions.device)
    return _fn()[1].apply(positions, e, F)
