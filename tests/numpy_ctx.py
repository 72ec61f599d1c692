"""A NumPy stand-in for the library's block operations (pwb200.Context
methods apply, kprec, gram, rotate, eigh, calc_grad, ortho_sqrt), with the
layouts of the C ABI: band-major (nb, Ngw) blocks, pw_gram writing A^H B
column-major, pw_rotate taking U column-major, pw_eigh returning
eigenvectors as rows.  Used by the CPU tests of the host compositions
(pwb200.davidson, pwb200.emin_pcg); test infrastructure only."""
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

    def calc_grad(self, ik, ispin, psi, Focc, wk):
        import torch
        from oracle import ops
        g = ops.calc_grad(self.H, psi.numpy().T, ik, np.asarray(Focc, dtype=np.float64), wk)
        return torch.from_numpy(np.ascontiguousarray(g.T))

    def ortho_sqrt(self, X):
        import torch
        from oracle.lobpcg import ortho_sqrt
        X.copy_(torch.from_numpy(np.ascontiguousarray(ortho_sqrt(X.numpy().T).T)))
