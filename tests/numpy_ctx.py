"""A NumPy stand-in for the library's block operations (pwb200.Context
methods apply, kprec, gram, rotate, eigh, calc_grad, ortho_sqrt), with the
layouts of the C ABI: band-major (nb, Ngw) blocks, pw_gram writing A^H B
column-major, pw_rotate taking U column-major, pw_eigh returning
eigenvectors as rows; SCFCtx adds pw_update's sums, calc_rhoe, band
energies and LOBPCG through the oracle, and HostHam the host attributes of
pwb200.Hamiltonian, so the SCF drivers run on the CPU.  Used by the CPU
tests of the host compositions and drivers; test infrastructure only."""
import numpy as np
import scipy.linalg as sla


class NumpyCtx:
    """The block operations diag_davidson_k uses, in NumPy on torch CPU tensors."""

    def __init__(self, H):
        self.H = H

    def apply(self, ik, ispin, psi, Hpsi):
        import torch
        from oracle import ops
        Hpsi.copy_(torch.from_numpy(np.ascontiguousarray(ops.op_H(self.H, psi.numpy().T, ik).T)))

    def kprec(self, ik, x, out):
        import torch
        from oracle import ops
        out.copy_(torch.from_numpy(np.ascontiguousarray(ops.Kprec(self.H, x.numpy().T, ik).T)))

    def gram(self, A, B, out, accumulate=False):
        import torch
        C = A.numpy().conj() @ B.numpy().T          # (m, n) = A^H B
        out.copy_(torch.from_numpy(np.ascontiguousarray(C.T)) + (out if accumulate else 0))

    def rotate(self, A, U, out, accumulate=False):
        import torch
        R = (A.numpy().T @ U.numpy().T).T           # (n, M) = (A U)^T
        out.copy_(torch.from_numpy(np.ascontiguousarray(R)) + (out if accumulate else 0))

    def eigh(self, T, G=None, k=None, vectors=True):
        import torch
        Tm = T.numpy().T
        Gm = G.numpy().T if G is not None else None
        k = Tm.shape[0] if k is None else k
        lam, S = sla.eigh(Tm, Gm, lower=False)
        Sv = torch.from_numpy(np.ascontiguousarray(S[:, :k].T)) if vectors else None
        return torch.from_numpy(lam[:k].copy()), Sv

    def chol_rinv(self, C):
        import torch
        from oracle.lobpcg import _chol_upper
        R = _chol_upper(C.numpy().T)
        return torch.from_numpy(np.ascontiguousarray(np.linalg.inv(R).T))

    def calc_grad(self, ik, ispin, psi, Focc, wk):
        import torch
        from oracle import ops
        g = ops.calc_grad(self.H, psi.numpy().T, ik, np.asarray(Focc, dtype=np.float64), wk)
        return torch.from_numpy(np.ascontiguousarray(g.T))

    def ortho_sqrt(self, X):
        import torch
        from oracle.lobpcg import ortho_sqrt
        X.copy_(torch.from_numpy(np.ascontiguousarray(ortho_sqrt(X.numpy().T).T)))


class SCFCtx(NumpyCtx):
    """NumpyCtx plus the density, update! and band-energy entry points."""
    torch_device = "cpu"
    device = 0

    def update(self, rho, Vps):
        from oracle import energies
        r = rho.numpy().copy()
        self.H.update(r)
        Eps, EH, Exc = energies.calc_E_local(self.H, r)
        dVol = self.H.pw.CellVolume / self.H.pw.Npoints
        return np.array([2.0 * EH / dVol, Eps / dVol, Exc / dVol])

    def mix_pulay(self, x, gx, beta, it, mixdim, clamp=True):
        """pw_mix_pulay through the oracle's mix_pulay (its history here)."""
        import torch
        from oracle.scf import mix_pulay
        if it == 1:
            n = x.numel()
            self._mix = (np.zeros((n, mixdim)), np.zeros((n, mixdim)), {})
        X, F, state = self._mix
        r = mix_pulay(x.numpy().copy(), gx.numpy().copy(), beta, X, F, it, mixdim, state)
        if clamp:
            r = np.maximum(r, np.finfo(np.float64).eps)
        x.copy_(torch.from_numpy(r))
        return x

    def lobpcg(self, ik, ispin, X, tol=1e-5, nitermax=100, nconv=0):
        import torch
        from oracle.lobpcg import diag_LOBPCG_k
        Xh = X.numpy().T.copy()
        ev = diag_LOBPCG_k(self.H, Xh, ik, tol=tol, NiterMax=nitermax, Nstates_conv=nconv)
        X.copy_(torch.from_numpy(np.ascontiguousarray(Xh.T)))
        return ev, 0

    def calc_rhoe(self, ik, psi, w, rho, accumulate=False):
        import torch
        from oracle import ops
        pw = self.H.pw
        psiks = [np.zeros((pw.gvecw.Ngw[k], psi.shape[0]), dtype=np.complex128) for k in range(pw.kpoints.Nkpt)]
        psiks[ik] = psi.numpy().T
        Focc = np.zeros((psi.shape[0], pw.kpoints.Nkpt))
        Focc[:, ik] = np.asarray(w) / pw.kpoints.wk[ik]
        r = torch.from_numpy(ops.calc_rhoe(self.H, psiks, Focc=Focc))
        if accumulate:
            rho.add_(r)
        else:
            rho.copy_(r)

    def band_energies(self, ik, psi, w):
        from oracle import ops
        p = psi.numpy().T
        Kp = np.zeros_like(p)
        ops.op_K(self.H, p, Kp, ik)
        Vp = np.zeros_like(p)
        ops.op_V_Ps_nloc(self.H, p, Vp, ik)
        w = np.asarray(w)
        return np.array([float(np.sum(w * np.real(np.sum(p.conj() * Kp, axis=0)))),
                         float(np.sum(w * np.real(np.sum(p.conj() * Vp, axis=0))))])


class HostHam:
    """The attributes of pwb200.Hamiltonian the driver reads, host-only."""

    def __init__(self, Ho, meshk):
        import pwb200
        from pwb200.system import kpoint_grid
        k, w = kpoint_grid(Ho.atoms.LatVecs, meshk)
        self.system = pwb200.System(["Si", "Si"], Ho.atoms.positions, Ho.atoms.LatVecs)
        self.basis = pwb200.Basis(Ho.atoms.LatVecs, 15.0, kpts=k)
        self.wk = w
        from oracle import systems
        self.pspots = [pwb200.GTH(systems.psp("Si-q4.gth"))]
        self.Zvals = np.array([4.0])
        self.Nelectrons = 8.0
        self.V_Ps_loc = Ho.V_Ps_loc
        self.sym = None
        self.ctx = SCFCtx(Ho)

    def setup_density(self):
        pass
