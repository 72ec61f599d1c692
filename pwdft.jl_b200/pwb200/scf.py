"""KS_solve_SCF! with every step of the SCF iteration on the device.

Mirrors KS_solve_SCF.jl:24-373 (Nspin = 1; simple density mixing by default,
as there, or Pulay; Fermi-Dirac smearing):
  ethr schedule            KS_solve_SCF.jl:177-185
  diag_LOBPCG!             pw_lobpcg per k-point          (device, update_psi="LOBPCG"), or
                           pw_lobpcg_multi for all k-points together (batched=True, nb <= 16)
  diag_davidson!           pwb200.davidson per k-point    (device, update_psi="davidson", FP64;
                           the 2-block solver KS_solve_SCF.jl:194-198 calls)
  diag_davidson_qe!        pw_davidson per k-point        (device, update_psi="davidson_qe";
                           the QE-style solver of electrons_scf.jl:150, FP64 or mixed)
  diag_CheFSI!             pwb200.chefsi per k-point      (device, update_psi="CheFSI",
                           cheby_degree; KS_solve_SCF.jl:205-208)
  diag_Emin_PCG!           pwb200.emin_pcg per k-point    (device, update_psi="PCG", FP64;
                           KS_solve_SCF.jl:199-203)
  calc_rhoe!               pw_calc_rhoe                   (device)
  symmetrize_rhoe!         pw_symmetrize_rhoe             (device, Hamiltonians built with symmetry)
  mix_pulay! / simple      mix_pulay.jl:1-41              (device: pw_mix_pulay, history in the library)
  smearing (use_smearing)  KS_solve_SCF.jl:218-223, occupations.jl:6-245  (host: Fermi level
                           by bisection over the Nstates x Nkpt eigenvalues, -TS)
  rho >= eps clamp         KS_solve_SCF.jl:277-281        (device)
  update!                  pw_update (Poisson, VWN, V_tot) (device)
  calc_energies            pw_update sums + pw_band_energies (device, FP64)
  convergence              |dE| < etot_conv_thr twice      (host scalar)
With a torch.distributed process group the k-points are shared out over the
ranks (pwb200.kshard): each rank solves and sums its own, and the density,
band energies and eigenvalues are all-reduced; psiks then holds this rank's
blocks only (None elsewhere).
The starting density (guess_rhoe.jl) and E_NN (Ewald) are computed once on
the host, as set-up.

precision = "fp64" runs the reference's FP64 path; "mixed" runs FP32
blocks with split-BF16x3 tensor-core contractions until |dE| stays below
`fp64_switch` for two iterations, then converts psi to complex128 and finishes in FP64
(iterative refinement; the Pulay history is kept: restarting it costs
more FP64 iterations than it saves).
"""
import time

import numpy as np

from .system import kpoint_grid, guess_rhoe, ewald_energy

EPS = np.finfo(np.float64).eps


def torch_device(ctx):
    """The torch device of a context's blocks: cuda:<device>, or the
    `torch_device` a host stand-in of the context declares (CPU tests)."""
    return getattr(ctx, "torch_device", None) or f"cuda:{ctx.device}"


def occupations(Nelectrons, Nstates, Nkpt):
    """Electrons.jl:120-262 for Nspin = 1 without smearing."""
    nocc = int(round(Nelectrons / 2))
    if nocc * 2 < Nelectrons:
        nocc += 1
    F = np.zeros((Nstates, Nkpt))
    F[:nocc - 1, :] = 2.0
    F[nocc - 1, :] = 1.0 if int(round(Nelectrons)) % 2 == 1 else 2.0
    return F, nocc


def fermi_dirac(x):
    """wgauss (occupations.jl:71-83): 1/(1 + e^-x), 0 below -200, 1 above 200."""
    with np.errstate(over="ignore"):
        f = 1.0 / (1.0 + np.exp(-x))
    return np.where(x < -200.0, 0.0, np.where(x > 200.0, 1.0, f))


def smeared_occupations(Nelectrons, wk, kT, evals):
    """calc_Focc + calc_entropy (occupations.jl:6-32, 126-192, 222-245),
    Nspin = 1: E_fermi by bisection of sum 2 wk f((E - evals)/kT) = Nelectrons
    between min(evals) - 2kT and max(evals) + 2kT (stop at |N - Nel| < 1e-10
    or a step below 1e-10, 300 steps at most); Focc = 2 f; mTS = sum 2 wk kT
    (f log f + (1 - f) log(1 - f)) over |x| <= 36.  Returns (Focc, E_fermi, mTS)."""
    wk = np.asarray(wk, dtype=np.float64)
    count = lambda E: float(np.sum(2.0 * wk * fermi_dirac((E - evals) / kT).sum(axis=0)))
    lo = evals[0, :].min() - 2 * kT
    hi = evals[-1, :].max() + 2 * kT
    eps = np.finfo(np.float64).eps
    if count(hi) - Nelectrons < -eps or count(lo) - Nelectrons > eps:
        raise ValueError("Bounds for E_fermi is not found")
    Ef = Ef_old = 0.5 * (lo + hi)
    for _ in range(300):
        n = count(Ef)
        if abs(n - Nelectrons) < 1e-10:
            break
        if n - Nelectrons < -1e-10:
            lo = Ef
        else:
            hi = Ef
        Ef = 0.5 * (lo + hi)
        if abs(Ef - Ef_old) < 1e-10:
            break
        Ef_old = Ef
    x = (Ef - evals) / kT
    Focc = 2.0 * fermi_dirac(x)
    ok = np.abs(x) <= 36.0
    f = 1.0 / (1.0 + np.exp(-np.where(ok, x, 0.0)))
    w1 = np.where(ok, f * np.log(f) + (1.0 - f) * np.log(1.0 - f), 0.0)
    mTS = float(np.sum(2.0 * wk[None, :] * kT * w1))
    return Focc, Ef, mTS


def rand_psiks(Ham, Nstates, seed, dtype, keep=None):
    """rand_BlochWavefunc (gen_wavefunc.jl:75-92): ortho_sqrt(rand(ComplexF64)),
    one seeded stream over all k-points; blocks outside `keep` are None."""
    import torch
    rng = np.random.default_rng(seed)
    out = []
    for ik in range(Ham.basis.Nkpt):
        ngw = Ham.basis.Ngw[ik]
        psi = rng.random((ngw, Nstates)) + 1j * rng.random((ngw, Nstates))
        if keep is not None and ik not in keep:
            out.append(None)
            continue
        w, U = np.linalg.eigh(psi.conj().T @ psi)
        psi = psi @ ((U / np.sqrt(w)) @ U.conj().T)
        out.append(torch.from_numpy(np.ascontiguousarray(psi.T)).to(torch_device(Ham.ctx)).to(dtype).contiguous())
    return out


def KS_solve_SCF(Ham, meshk=None, Nstates=None, betamix=0.2, mix_method="simple", mixdim=5, etot_conv_thr=1e-6,
                 ethr_evals_last=1e-5, NiterMax=100, precision="fp64", fp64_switch=1e-5, seed=1234, psiks=None,
                 verbose=False, lobpcg_maxiter=100, update_psi="LOBPCG", use_smearing=False, kT=1e-3,
                 savewfc=False, wfc_dir=".", batched=False, cheby_degree=8):
    """Runs the SCF loop; returns a dict with energies, eigenvalues, timings
    and the per-iteration log."""
    import torch
    ctx = Ham.ctx
    b = Ham.basis
    dev = torch_device(ctx)

    def sync():
        if dev.startswith("cuda"):
            torch.cuda.synchronize()
    N = b.Npoints
    dVol = b.CellVolume / N
    Nel = Ham.Nelectrons
    if Nstates is None:
        Nstates = int(round(Nel / 2)) + (1 if int(round(Nel)) % 2 else 0)
    Focc, Nocc = occupations(Nel, Nstates, b.Nkpt)
    wk = Ham.wk
    Ham.setup_density()
    if update_psi not in ("LOBPCG", "davidson", "davidson_qe", "CheFSI", "PCG"):
        raise ValueError("update_psi must be 'LOBPCG', 'davidson', 'davidson_qe', 'CheFSI' or 'PCG'")
    if mix_method not in ("simple", "pulay"):
        # KS_solve_SCF.jl:240-272 also has linear_adaptive, broyden, rpulay,
        # ppulay and anderson, and raises on any other name
        raise ValueError("mix_method must be 'simple' or 'pulay' (the reference's linear_adaptive, broyden, "
                         "rpulay, ppulay and anderson mixers are not built)")
    if update_psi == "PCG" and precision != "fp64":
        raise ValueError("update_psi='PCG' (diag_Emin_PCG!) runs on FP64 blocks only")
    if update_psi == "davidson" and precision != "fp64":
        raise ValueError("update_psi='davidson' (the 2-block diag_davidson!) runs on FP64 blocks only; "
                         "update_psi='davidson_qe' has a mixed-precision path")
    crng = np.random.default_rng(seed + 1)   # Lanczos start vectors of CheFSI
    mixed = precision == "mixed"
    dt = torch.complex64 if mixed else torch.complex128
    from .kshard import make_shards
    shards = make_shards(b.Ngw, Nstates)
    gamma = shards.kind == "gamma"
    if gamma and update_psi != "LOBPCG":
        raise ValueError("Gamma-point sharding over ranks runs update_psi='LOBPCG' only")
    mine = shards.mine
    from .gshard import split
    ba, bb = split(Nstates, shards.world)[shards.rank] if gamma else (0, Nstates)
    if savewfc and shards.world > 1:
        raise ValueError("savewfc with k-point sharding: write each rank's blocks with pwb200.io instead")
    if psiks is None:
        psiks = rand_psiks(Ham, Nstates, seed, dt, keep=set(mine))
    else:
        psiks = [p.to(dt).contiguous() if (p is not None and ik in mine) else None for ik, p in enumerate(psiks)]
    Vps = torch.from_numpy(Ham.V_Ps_loc).to(dev)
    rho = torch.from_numpy(guess_rhoe(Ham.system, b, Ham.pspots, Nel)).to(dev)
    ctx.update(rho, Vps)
    E_NN = ewald_energy(Ham.system.LatVecs, Ham.system.positions, Ham.Zvals[Ham.system.atm2species])
    rho_new = torch.zeros(N, dtype=torch.float64, device=dev)
    Etot_old, Nconv, ethr = 0.0, 0, 0.1
    imix = 0
    nsw = 0   # consecutive iterations with |dE| below fp64_switch (as the convergence test)
    log = []
    evals = np.zeros((Nstates, b.Nkpt))
    t_start = time.perf_counter()
    t_diag = t_rho = t_upd = 0.0
    switched_at = None
    E_fermi = None
    E = {}
    for it in range(1, NiterMax + 1):
        ethr = 0.1 if it == 1 else (0.01 if it == 2 else max(ethr / 5.0, ethr_evals_last))
        t0 = time.perf_counter()
        nit = [0]
        evals[:] = 0.0
        if gamma:
            # one k-point, its work split over the ranks (pwb200.gshard)
            from .gshard import diag_LOBPCG_gamma
            ev, n = diag_LOBPCG_gamma(ctx, psiks[0], shards, tol=ethr, NiterMax=lobpcg_maxiter, Nstates_conv=Nocc)
            evals[:, 0] = ev
            nit.append(n)
        elif batched and update_psi == "LOBPCG" and mine:
            # every k-point of this rank advanced together (pw_lobpcg_multi)
            ev, n = ctx.lobpcg_multi(mine, 0, [psiks[ik] for ik in mine], tol=ethr, nitermax=lobpcg_maxiter, nconv=Nocc)
            evals[:, mine] = ev
            nit.append(n)
        for ik in ([] if (gamma or (batched and update_psi == "LOBPCG")) else mine):
            if update_psi == "LOBPCG":
                ev, n = ctx.lobpcg(ik, 0, psiks[ik], tol=ethr, nitermax=lobpcg_maxiter, nconv=Nocc)
            elif update_psi == "davidson":
                from .davidson import diag_davidson_k
                ev, n = diag_davidson_k(ctx, ik, 0, psiks[ik], tol=ethr, NiterMax=lobpcg_maxiter, Nstates_conv=Nocc)
            elif update_psi == "davidson_qe":
                ev, n = ctx.davidson(ik, 0, psiks[ik], tol=ethr, nitermax=lobpcg_maxiter)
            elif update_psi == "PCG":
                from .emin_pcg import diag_Emin_PCG_k
                ev, n = diag_Emin_PCG_k(ctx, ik, 0, psiks[ik], tol=ethr, NiterMax=lobpcg_maxiter, Nstates_conv=Nocc)
            else:
                from .chefsi import diag_chefsi_k
                ev, n = diag_chefsi_k(ctx, ik, 0, psiks[ik], cheby_degree, crng), 0
            evals[:, ik] = ev
            nit.append(n)
        if shards.world > 1:
            shards.reduce_evals(evals)
        sync()
        mTS = 0.0
        if use_smearing:
            Focc, E_fermi, mTS = smeared_occupations(Nel, wk, kT, evals)
        t1 = time.perf_counter()
        rho_new.zero_()
        for j, ik in enumerate(mine):
            if bb > ba:
                ctx.calc_rhoe(ik, psiks[ik][ba:bb], wk[ik] * Focc[ba:bb, ik], rho_new, accumulate=(j > 0))
        shards.sum_(rho_new)
        if Ham.sym is not None:
            ctx.symmetrize_rhoe(rho_new)
        diffRhoe = float(torch.sum(torch.abs(rho_new - rho)).item()) / N
        sync()
        t2 = time.perf_counter()
        imix += 1
        if mix_method == "pulay":
            rho = ctx.mix_pulay(rho, rho_new, betamix, imix, mixdim, clamp=True)
        else:
            rho = torch.clamp(betamix * rho_new + (1 - betamix) * rho, min=EPS)
        sums = ctx.update(rho, Vps)
        Ek = En = 0.0
        for ik in mine:
            if bb > ba:
                e2 = ctx.band_energies(ik, psiks[ik][ba:bb], wk[ik] * Focc[ba:bb, ik])
                Ek += e2[0]
                En += e2[1]
        if shards.world > 1:
            Ek, En = [float(v) for v in shards.sum_(torch.tensor([Ek, En], dtype=torch.float64, device=dev)).tolist()]
        E = {"Kinetic": Ek, "Ps_loc": sums[1] * dVol, "Ps_nloc": En, "Hartree": 0.5 * sums[0] * dVol,
             "XC": sums[2] * dVol, "NN": E_NN, "mTS": mTS}
        E["Total"] = sum(E.values())
        t3 = time.perf_counter()
        t_diag += t1 - t0
        t_rho += t2 - t1
        t_upd += t3 - t2
        diffE = abs(E["Total"] - Etot_old)
        nit = np.array(nit)
        log.append((it, E["Total"], diffE, diffRhoe, int(np.max(nit % 1000)), "c64" if mixed else "c128",
                    int(np.sum(nit // 1000))))
        if verbose:
            print("SCF: %5d %18.10f %12.5e %12.5e  %s  %s its %d restarts %d  ethr %.1e  %.2fs" % (
                it, E["Total"], diffE, diffRhoe, log[-1][5], update_psi, log[-1][4], log[-1][6], ethr, t1 - t0),
                flush=True)
        Nconv = Nconv + 1 if diffE < etot_conv_thr else 0
        if Nconv >= 2:
            break
        nsw = nsw + 1 if diffE < fp64_switch else 0
        if mixed and nsw >= 2 and it > 2:
            # iterative refinement: finish in FP64
            psiks = [p.to(torch.complex128).contiguous() if p is not None else None for p in psiks]
            mixed = False
            switched_at = it
        Etot_old = E["Total"]
    sync()
    if savewfc:
        # KS_solve_SCF_potmix.jl:301-307: WFC_ikspin_<n>.data per (k-point, spin)
        from .io import write_psiks
        write_psiks(psiks, wfc_dir)
    return {"energies": E, "evals": evals, "Focc": Focc, "E_fermi": E_fermi, "iterations": len(log), "log": log,
            "time_s": time.perf_counter() - t_start,
            "time_diag_s": t_diag, "time_rhoe_s": t_rho, "time_update_s": t_upd, "switched_to_fp64_at": switched_at,
            "psiks": psiks, "rho": rho, "kpoints_local": mine}
