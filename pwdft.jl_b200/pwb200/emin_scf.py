"""KS_solve_Emin_PCG! (KS_solve_Emin_PCG.jl:27-270): direct minimisation of the
Kohn-Sham energy by preconditioned conjugate gradients (Ismail-Beigi and
Arias), Nspin = 1, every step on the device:

  starting density, update!        guess_rhoe (host set-up), pw_update
  initial diag_LOBPCG! (10 its)    pw_lobpcg per k-point (unless skipped)
  calc_grad with occupations       pw_calc_grad (w_k f_i)
  Kprec                            pw_kprec
  beta, alpha dot products         real traces of pw_gram (FP64)
  trial point, update              ortho_sqrt (pw_ortho_sqrt) of psi + a d
  trial and new densities          pw_calc_rhoe (+ pw_symmetrize_rhoe), pw_update
  energies                         pw_update sums + pw_band_energies
  final Rayleigh-Ritz rotation     pw_apply + pw_gram, pw_eigh, pw_rotate

The search directions and trial points are elementwise tensor updates; the
per-k-point scalars are host FP64.  FP64 blocks (the reference's precision).
"""
import time

import numpy as np

from .scf import occupations, rand_psiks, torch_device
from .system import guess_rhoe, ewald_energy
from .emin_pcg import _rtrace, _ortho, _rayleigh


def _density(Ham, psis, Focc, wk, rho):
    ctx = Ham.ctx
    for ik, psi in enumerate(psis):
        ctx.calc_rhoe(ik, psi, wk[ik] * Focc[:, ik], rho, accumulate=(ik > 0))
    if getattr(Ham, "sym", None) is not None:
        ctx.symmetrize_rhoe(rho)
    return rho


def _energies(Ham, psis, Focc, wk, sums, dVol, E_NN):
    Ek = En = 0.0
    for ik, psi in enumerate(psis):
        e2 = Ham.ctx.band_energies(ik, psi, wk[ik] * Focc[:, ik])
        Ek += e2[0]
        En += e2[1]
    E = {"Kinetic": Ek, "Ps_loc": sums[1] * dVol, "Ps_nloc": En, "Hartree": 0.5 * sums[0] * dVol,
         "XC": sums[2] * dVol, "NN": E_NN, "mTS": 0.0}
    E["Total"] = sum(E.values())
    return E


def KS_solve_Emin_PCG(Ham, psiks=None, alpha_t=3e-5, NiterMax=200, i_cg_beta=2, etot_conv_thr=1e-6,
                      skip_initial_diag=False, alpha_max=2.1, restrict_linmin=False, Nstates=None, seed=1234,
                      verbose=False):
    """Returns a dict with energies, eigenvalues (Nstates, Nkpt), iterations
    and the per-step log (iter, Etot, dE); psiks (list of complex128
    (Nstates, Ngw) device blocks, or None for the seeded random start) ends
    as the Ritz vectors."""
    import torch
    ctx = Ham.ctx
    b = Ham.basis
    dev = torch_device(ctx)
    N = b.Npoints
    dVol = b.CellVolume / N
    Nel = Ham.Nelectrons
    Nkpt = b.Nkpt
    if Nstates is None:
        Nstates = int(round(Nel / 2)) + (1 if int(round(Nel)) % 2 else 0)
    Focc, _ = occupations(Nel, Nstates, Nkpt)
    wk = Ham.wk
    Ham.setup_density()
    if psiks is None:
        psiks = rand_psiks(Ham, Nstates, seed, torch.complex128)
    if any(p.dtype != torch.complex128 for p in psiks):
        raise TypeError("KS_solve_Emin_PCG runs on complex128 blocks (the reference's FP64 path)")
    Vps = torch.from_numpy(np.asarray(Ham.V_Ps_loc, dtype=np.float64)).to(dev)
    rho = torch.from_numpy(guess_rhoe(Ham.system, b, Ham.pspots, Nel)).to(dev)       # :65-71
    sums = ctx.update(rho, Vps)                                                        # :73
    if not skip_initial_diag:                                                          # :75-79
        for ik in range(Nkpt):
            ctx.lobpcg(ik, 0, psiks[ik], tol=1e-5, nitermax=10)
    E_NN = ewald_energy(Ham.system.LatVecs, Ham.system.positions, Ham.Zvals[Ham.system.atm2species])
    E = _energies(Ham, psiks, Focc, wk, sums, dVol, E_NN)                              # :97-101
    g, Kg, d = [None] * Nkpt, [None] * Nkpt, [None] * Nkpt
    g_old = [torch.zeros_like(p) for p in psiks]
    d_old = [torch.zeros_like(p) for p in psiks]
    Kg_old = [torch.zeros_like(p) for p in psiks]
    psic = [None] * Nkpt
    beta = np.zeros(Nkpt)
    alpha = np.zeros(Nkpt)
    Etot_old = 0.0
    Nconverges = 0
    log = []
    t0 = time.perf_counter()
    it = 0
    for it in range(1, NiterMax + 1):
        for i in range(Nkpt):                                                          # :130-179
            g[i] = ctx.calc_grad(i, 0, psiks[i], Focc[:, i], wk[i])
            Kg[i] = torch.empty_like(g[i])
            ctx.kprec(i, g[i], Kg[i])
            if it != 1:
                gK, goK = _rtrace(ctx, g[i], Kg[i]), _rtrace(ctx, g_old[i], Kg[i])
                if i_cg_beta == 1:
                    beta[i] = gK / _rtrace(ctx, g_old[i], Kg_old[i])
                    if abs(beta[i] - 1.0) < 0.2:
                        beta[i] = 0.0
                elif i_cg_beta == 2:
                    beta[i] = (gK - goK) / _rtrace(ctx, g_old[i], Kg_old[i])
                elif i_cg_beta == 3:
                    beta[i] = (gK - goK) / (_rtrace(ctx, g[i], d[i]) - _rtrace(ctx, g_old[i], d[i]))
                else:
                    beta[i] = gK / (_rtrace(ctx, d_old[i], g[i]) - _rtrace(ctx, d_old[i], g_old[i]))
                    if abs(beta[i] - 1.0) < 0.2:
                        beta[i] = 0.0
            if beta[i] < 0.0 or np.isnan(beta[i]):
                beta[i] = 0.0
            d[i] = torch.add(torch.neg(Kg[i]), d_old[i], alpha=float(beta[i]))
            psic[i] = _ortho(ctx, torch.add(psiks[i], d[i], alpha=alpha_t))
        rho_t = torch.zeros(N, dtype=torch.float64, device=dev)                        # :181-183
        ctx.update(_density(Ham, psic, Focc, wk, rho_t), Vps)
        for i in range(Nkpt):                                                          # :185-207
            gt = ctx.calc_grad(i, 0, psic[i], Focc[:, i], wk[i])
            gd = _rtrace(ctx, g[i], d[i])
            denum = gd - _rtrace(ctx, gt, d[i])
            alpha[i] = abs(alpha_t * gd / denum) if denum != 0.0 else 0.0
            if restrict_linmin and alpha[i] > alpha_max:
                alpha[i] = alpha_max
            psiks[i].copy_(_ortho(ctx, torch.add(psiks[i], d[i], alpha=float(alpha[i]))))
        rho = _density(Ham, psiks, Focc, wk, torch.zeros(N, dtype=torch.float64, device=dev))   # :209-214
        sums = ctx.update(rho, Vps)
        E = _energies(Ham, psiks, Focc, wk, sums, dVol, E_NN)
        diffE = Etot_old - E["Total"]
        log.append((it, E["Total"], diffE))
        if verbose:
            print("Emin_PCG step %4d = %18.10f %16.6e" % (it, E["Total"], diffE), flush=True)
        Nconverges = Nconverges + 1 if abs(diffE) < etot_conv_thr else 0               # :226-238
        if Nconverges >= 2:
            break
        g_old, d_old, Kg_old = list(g), list(d), list(Kg)
        Etot_old = E["Total"]
    evals = np.zeros((Nstates, Nkpt))                                                  # :247-256
    for i in range(Nkpt):
        _ortho(ctx, psiks[i])
        lam, S = _rayleigh(ctx, i, 0, psiks[i], True)
        Xn = torch.zeros_like(psiks[i])
        ctx.rotate(psiks[i], S, Xn)
        psiks[i].copy_(Xn)
        evals[:, i] = lam
    return {"energies": E, "evals": evals, "iterations": it, "log": log, "psiks": psiks,
            "time_s": time.perf_counter() - t0, "rho": rho}
