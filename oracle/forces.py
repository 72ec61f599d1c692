"""Ionic forces (Hartree/bohr).

Oracle (test infrastructure only).  Restates PWDFT.jl:
  calc_forces_Ps_loc.jl:13-71      local pseudopotential force
  calc_forces_Ps_nloc.jl:291-343   GTH nonlocal force
  calc_forces_Ps_nloc.jl:347-411   dbetaNL = i (G+k) betaNL and its projections
  calc_forces_NN.jl:1-142          Ewald (ion-ion) force
  calc_forces.jl:1-17              the sum (no symmetrisation: use_symmetry=false,
                                   no NLCC, no SCF correction for GTH)
"""
import numpy as np
from scipy.special import erfc

from .gth import eval_Vloc_G
from .ham import R_to_G
from .ops import calc_betaNL_psi


def calc_forces_Ps_loc(Ham, Rhoe):
    """calc_forces_Ps_loc.jl:13-71: F_a = sum_{G != 0} Re(i G V_sp(G) conj(rho(G)) e^{-i G.tau_a}),
    rho(G) = fft(rho)/N; V_sp(G) per G-shell without the 1/Omega (it cancels)."""
    pw, atoms = Ham.pw, Ham.atoms
    N = pw.Npoints
    RhoeG = R_to_G(pw.Ns, np.asarray(Rhoe, dtype=np.complex128)) / N
    G = pw.gvec.G
    rG = RhoeG[pw.gvec.idx_g2r]
    Vgl = [eval_Vloc_G(psp, pw.gvec.G2_shells) for psp in Ham.pspots]
    F = np.zeros((3, atoms.Natoms))
    for ia in range(atoms.Natoms):
        isp = atoms.atm2species[ia]
        tau = atoms.positions[:, ia]
        GX = tau @ G
        Sf = np.cos(GX) - 1j * np.sin(GX)
        w = Vgl[isp][pw.gvec.idx_g2shells] * np.conj(rG) * Sf
        w[0] = 0.0                                  # G = 0 (sorted first) skipped
        F[:, ia] = np.real(1j * (G * w[None, :])).sum(axis=1)
    return F


def beta_atom(Ham):
    """Atom of each projector (prj2beta order: atom, l, m, projector)."""
    at = np.zeros(Ham.NbetaNL, dtype=np.int64)
    for (iprj, ia, l, m), ib in Ham.prj2beta.items():
        at[ib] = ia
    return at


def calc_dbetaNL_psi(Ham, psi, ik):
    """calc_forces_Ps_nloc.jl:347-411: dB[d, ist, jb] = dot(i g_d betaNL[:, jb], psi[:, ist])
    = -i sum_g g_d conj(betaNL[g, jb]) psi[g, ist]  (g = G + k)."""
    pw = Ham.pw
    idx = pw.gvecw.idx_gw2g[ik]
    g = pw.gvec.G[:, idx] + pw.kpoints.k[:, ik][:, None]
    beta = Ham.betaNL[ik]
    dB = np.zeros((3, psi.shape[1], beta.shape[1]), dtype=np.complex128)
    for d in range(3):
        # dot(a, b) = a^H b:  (i g_d beta)^H psi -> (Nbeta, Nstates), stored [ist, jb]
        dB[d] = ((1j * g[d][:, None] * beta).conj().T @ psi).T
    return dB


def calc_forces_Ps_nloc(Ham, psiks):
    """calc_forces_Ps_nloc.jl:291-343: F_a += 2 wk f Re(h_ij conj(B_i) dB_j) over the
    (ibeta, jbeta, h_ij) pairs of atom a."""
    F = np.zeros((3, Ham.atoms.Natoms))
    if Ham.NbetaNL == 0:
        return F
    at = beta_atom(Ham)
    trip = np.array([(ib, jb) for ib, jb, h in Ham.nl_triplets], dtype=np.int64)
    hh = np.array([h for ib, jb, h in Ham.nl_triplets])
    for ik, psi in enumerate(psiks):
        B = calc_betaNL_psi(Ham, psi, ik)           # (Nstates, Nbeta)
        dB = calc_dbetaNL_psi(Ham, psi, ik)         # (3, Nstates, Nbeta)
        w = 2.0 * Ham.pw.kpoints.wk[ik] * Ham.Focc[:, ik]
        # per pair: sum over states of w_s Re(h conj(B[s, ib]) dB[:, s, jb])
        t = np.real(np.conj(B[:, trip[:, 0]])[None, :, :] * dB[:, :, trip[:, 1]])   # (3, Nstates, Npairs)
        contrib = np.einsum("s,dsp->dp", w, t) * hh[None, :]
        np.add.at(F.T, at[trip[:, 0]], contrib.T)
    return F


def _Herfc(x):
    return -2.0 * np.exp(-x * x) / np.sqrt(np.pi) - erfc(x) / x


def calc_forces_NN(Ham):
    """calc_forces_NN.jl:1-142: Ewald force with the reference's alpha search
    (G2_max = ecutrho) and real-space image range (ebsl = 1e-10)."""
    pw, atoms = Ham.pw, Ham.atoms
    tau = atoms.positions
    Z = Ham.Zvals[atoms.atm2species]
    Omega = pw.CellVolume
    charge = float(Z.sum())
    G2_max = pw.ecutrho
    alpha = 1.0
    ub = charge ** 2 * np.sqrt(alpha / np.pi) * erfc(np.sqrt(G2_max / 2.0 / alpha))
    while ub > 1e-6:
        alpha -= 0.1
        if alpha <= 0.0:
            raise ValueError("optimal alpha not found")
        ub = charge ** 2 * np.sqrt(alpha / np.pi) * erfc(np.sqrt(G2_max / 2.0 / alpha))
    G, G2 = pw.gvec.G[:, 1:], pw.gvec.G2[1:]
    GX = tau.T @ G                                   # (Natoms, Ng-1)
    aux = (Z[:, None] * (np.cos(GX) + 1j * np.sin(GX))).sum(axis=0)
    aux = aux * np.exp(-G2 / alpha / 4.0) / G2
    sumnb = np.cos(GX) * aux.imag[None, :] - np.sin(GX) * aux.real[None, :]
    F_G = (sumnb @ G.T).T * (-4.0 * np.pi * Z[None, :] / Omega)
    # real-space sum
    L = pw.LatVecs
    eta = np.sqrt(alpha)
    tmax = np.sqrt(0.5 * -np.log(1e-10)) / eta
    mm = [int(round(tmax / np.linalg.norm(L[:, i]) + 1.5)) for i in range(3)]
    ii, jj, kk = np.meshgrid(*[np.arange(-m, m + 1) for m in mm], indexing="ij")
    T = np.outer(L[:, 0], ii.ravel()) + np.outer(L[:, 1], jj.ravel()) + np.outer(L[:, 2], kk.ravel())
    F_R = np.zeros((3, atoms.Natoms))
    for ia in range(atoms.Natoms):
        for ja in range(ia + 1, atoms.Natoms):
            D = (tau[:, ia] - tau[:, ja])[:, None] - T
            D2 = (D * D).sum(axis=0)
            Dm = np.sqrt(D2)
            df = (eta * _Herfc(eta * Dm) / D2 * Z[ia] * Z[ja])[None, :] * D
            s = df.sum(axis=1)
            F_R[:, ia] -= s
            F_R[:, ja] += s
    return F_G + F_R


def calc_forces(Ham, psiks, Rhoe):
    """calc_forces.jl:1-17 for GTH: F_NN + F_Ps_loc + F_Ps_nloc, the nonlocal
    part symmetrised when the Hamiltonian uses symmetry (calc_forces.jl:11)."""
    F_nl = calc_forces_Ps_nloc(Ham, psiks)
    sym = getattr(Ham, "sym", None)
    if sym is not None and sym.Nsyms > 1:
        from .symmetry import symmetrize_vector
        F_nl = symmetrize_vector(Ham.atoms.LatVecs, sym, F_nl)
    return calc_forces_NN(Ham) + calc_forces_Ps_loc(Ham, Rhoe) + F_nl
