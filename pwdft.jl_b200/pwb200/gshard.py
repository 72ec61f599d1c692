"""Gamma-point sharding of the SCF over ranks (one process per GPU).

With a single k-point there is nothing to share out by k (pwb200.kshard), so
the work of one k-point is split (the exchanges are torch.distributed
collectives over the default group: NCCL between GPUs):

  op_H (op_H.jl:53-63)          by bands: rank r applies H to its contiguous
                                slice of the block's columns, then the slices
                                are all-gathered
  calc_rhoe (calc_rhoe.jl:51-78),
  band energies                 by bands, then an all-reduce of rho(r) / of
                                the two sums
  Rayleigh-Ritz Grams           by plane-wave rows: each rank forms A^H B over
  (diag_LOBPCG.jl:85,144,       its slice of the Ngw rows, then an all-reduce
  152-153,183-184)              of the (3 nb)^2 matrix
  rotations Q U                 by plane-wave rows, then an all-gather of the
  (diag_LOBPCG.jl:188-194)      rows
  small FP64 problems           solved on the device of rank 0 (pw_eigh,
  (eigen, cholesky)             pw_chol_rinv) and broadcast, so that every rank
                                continues from bit-identical matrices

Every rank holds the full blocks X, W, P (replicated) and takes the same
steps in the same order.  diag_LOBPCG_gamma follows diag_LOBPCG.jl:51-225
step for step (the FP64 algorithm of the reference, lock branch included).
"""
import numpy as np

EPS = np.finfo(np.float64).eps


def split(n, world):
    """Contiguous near-equal [start, stop) slices of range(n), one per rank."""
    q, r = divmod(n, world)
    out, s = [], 0
    for i in range(world):
        e = s + q + (1 if i < r else 0)
        out.append((s, e))
        s = e
    return out


class GammaShards:
    """Slices and collectives of one Gamma-point SCF.  world = 1 (no process
    group) runs the same code with every slice the whole range."""

    kind = "gamma"

    def __init__(self):
        import torch.distributed as dist
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.world = self.dist.get_world_size() if self.dist else 1
        self.rank = self.dist.get_rank() if self.dist else 0
        # gloo moves host tensors: device tensors are staged through the host
        self.stage = self.dist is not None and self.dist.get_backend() == "gloo"
        self.mine = [0]

    # ------------------------------------------------------------ collectives
    def _run(self, fn, t):
        if self.dist is None:
            return t
        if self.stage and t.is_cuda:
            h = t.cpu()
            fn(h)
            t.copy_(h)
        else:
            fn(t)
        return t

    def sum_(self, t):
        """In-place sum over ranks."""
        return self._run(lambda x: self.dist.all_reduce(x), t)

    def bcast_(self, t):
        """In place: rank 0's values on every rank."""
        return self._run(lambda x: self.dist.broadcast(x, 0), t)

    def reduce_evals(self, evals):
        """Every rank already holds all eigenvalues of the Gamma point."""
        return evals

    def gather_rows_(self, Y, sl):
        """Y (n, K): each rank filled Y[sl[rank][0]:sl[rank][1]] of dim 0;
        afterwards every rank holds all of Y."""
        if self.dist is None:
            return Y
        import torch
        w = max(b - a for a, b in sl)
        dev = "cpu" if self.stage else Y.device
        a, b = sl[self.rank]
        mine = torch.zeros((w,) + tuple(Y.shape[1:]), dtype=Y.dtype, device=dev)
        mine[:b - a] = Y[a:b].to(dev)
        parts = [torch.empty_like(mine) for _ in range(self.world)]
        self.dist.all_gather(parts, mine)
        for q, (a, b) in enumerate(sl):
            if q != self.rank and b > a:
                Y[a:b].copy_(parts[q][:b - a])
        return Y

    def gather_cols_(self, Y, sl):
        """Y (n, K): each rank filled the columns Y[:, sl[rank][0]:sl[rank][1]];
        afterwards every rank holds all of Y."""
        if self.dist is None:
            return Y
        import torch
        w = max(b - a for a, b in sl)
        dev = "cpu" if self.stage else Y.device
        a, b = sl[self.rank]
        mine = torch.zeros((Y.shape[0], w), dtype=Y.dtype, device=dev)
        mine[:, :b - a] = Y[:, a:b].to(dev)
        parts = [torch.empty_like(mine) for _ in range(self.world)]
        self.dist.all_gather(parts, mine)
        for q, (a, b) in enumerate(sl):
            if q != self.rank and b > a:
                Y[:, a:b].copy_(parts[q][:, :b - a])
        return Y


class GammaOps:
    """The block operations of diag_LOBPCG on replicated blocks (nb, Ngw),
    their work split over the ranks.  Matrices are in math convention
    (M[i, j]); the conversions to the C ABI's column-major storage happen
    here."""

    def __init__(self, ctx, ik, sh, ngw):
        self.ctx, self.ik, self.sh = ctx, ik, sh
        self.rows = split(ngw, sh.world)
        self.ngw = ngw

    def H(self, V):
        """op_H of every column of V, by band slices + all-gather."""
        import torch
        HV = torch.zeros_like(V)
        sl = split(V.shape[0], self.sh.world)
        a, b = sl[self.sh.rank]
        if b > a:
            self.ctx.apply(self.ik, 0, V[a:b], HV[a:b])
        return self.sh.gather_rows_(HV, sl)

    def kprec(self, R):
        import torch
        W = torch.empty_like(R)
        self.ctx.kprec(self.ik, R, W)
        return W

    def gram(self, A, B):
        """A^H B (m x n, complex128) over this rank's plane-wave rows, summed."""
        import torch
        a, b = self.rows[self.sh.rank]
        out = torch.zeros((B.shape[0], A.shape[0]), dtype=torch.complex128, device=A.device)
        if b > a:
            self.ctx.gram(A[:, a:b], B[:, a:b], out)
        self.sh.sum_(out)
        return out.T.contiguous()

    def rot(self, A, U, out=None, accumulate=False):
        """out (n, Ngw) (+)= the block A (k, Ngw) times U (k x n), by rows + all-gather."""
        import torch
        if out is None:
            out = torch.zeros((U.shape[1], A.shape[1]), dtype=A.dtype, device=A.device)
        a, b = self.rows[self.sh.rank]
        if b > a:
            self.ctx.rotate(A[:, a:b], U.T.contiguous(), out[:, a:b], accumulate=accumulate)
        return self.sh.gather_cols_(out, self.rows)

    def _small(self, fn, shapes, dtypes, device):
        """fn() on rank 0 (device solvers), its results broadcast."""
        import torch
        if self.sh.rank == 0:
            res = [r.contiguous() for r in fn()]
        else:
            res = [torch.empty(s, dtype=d, device=device) for s, d in zip(shapes, dtypes)]
        for r in res:
            self.sh.bcast_(r)
        return res

    def eigh(self, T, G=None, k=None, vectors=True):
        """Lowest k eigenpairs of Hermitian(T) (, Hermitian(G)) (upper
        triangles): (lam (k,), S (n x k))."""
        import torch
        n = T.shape[0]
        k = n if k is None else k

        def solve():
            Tt = T.T.contiguous()
            Gt = G.T.contiguous() if G is not None else None
            lam, S = self.ctx.eigh(Tt, Gt, k=k, vectors=vectors)
            return [lam] + ([S.T] if vectors else [])
        shapes = [(k,)] + ([(n, k)] if vectors else [])
        dtypes = [torch.float64] + ([torch.complex128] if vectors else [])
        res = self._small(solve, shapes, dtypes, T.device)
        return (res[0], res[1]) if vectors else (res[0], None)

    def chol_rinv(self, C):
        """inv(cholesky(Hermitian(C)).U) (n x n)."""
        import torch
        n = C.shape[0]
        return self._small(lambda: [self.ctx.chol_rinv(C.T.contiguous()).T], [(n, n)], [torch.complex128],
                           C.device)[0]


def diag_LOBPCG_gamma(ctx, X, sh, ik=0, tol=1e-5, NiterMax=100, Nstates_conv=0):
    """diag_LOBPCG!(Ham, X; tol, NiterMax, Nstates_conv) (diag_LOBPCG.jl:51-225)
    with its work split over the ranks of `sh` (GammaShards).  X (nb, Ngw)
    device block, the same on every rank, is overwritten with the Ritz
    vectors; returns (evals (nb,) numpy, iterations)."""
    import torch
    ops = GammaOps(ctx, ik, sh, X.shape[1])
    n = X.shape[0]
    if Nstates_conv == 0:
        Nstates_conv = n
    SMALL = 10.0 * EPS
    HX = ops.H(X)
    P = torch.zeros_like(X)
    HP = torch.zeros_like(X)
    evals_old = np.zeros(n)
    niter = 0
    cdt = X.dtype
    for it in range(1, NiterMax + 1):
        niter = it
        XHX = ops.gram(X, HX)
        lam, _ = ops.eigh(XHX, vectors=False)
        evals = lam.cpu().numpy()
        devals = np.abs(evals - evals_old)
        evals_old = evals.copy()
        R = HX.clone()
        ops.rot(X, -XHX.to(torch.complex128), out=R, accumulate=True)       # R = HX - X XHX
        nconv = int(np.sum(devals < tol))
        ilock = np.nonzero(devals <= SMALL)[0]
        iact = np.nonzero(devals > SMALL)[0]
        if nconv >= Nstates_conv:
            break
        W = ops.kprec(R)
        if len(ilock) > 0:
            il = torch.as_tensor(ilock, device=X.device)
            ia = torch.as_tensor(iact, device=X.device)
            Xlock = X.index_select(0, il)
            Xa = X.index_select(0, ia)
            Xa = ops.rot(Xlock, -ops.gram(Xlock, Xa), out=Xa.clone(), accumulate=True)
            Wa = W.index_select(0, ia)
            Wa = ops.rot(Xlock, -ops.gram(Xlock, Wa), out=Wa.clone(), accumulate=True)
            HXa = ops.H(Xa)
            HW = ops.H(Wa)
            HXa = ops.rot(Xlock, -ops.gram(Xlock, HXa), out=HXa.clone(), accumulate=True)
            HW = ops.rot(Xlock, -ops.gram(Xlock, HW), out=HW.clone(), accumulate=True)
            Rinv = ops.chol_rinv(ops.gram(Wa, Wa))
            Wa = ops.rot(Wa, Rinv)
            HW = ops.rot(HW, Rinv)
            Q = torch.cat([Xa, Wa])
            HQ = torch.cat([HXa, HW])
            _, S = ops.eigh(ops.gram(Q, HQ), ops.gram(Q, Q), k=len(iact))
            Xact = ops.rot(Q, S)
            X.copy_(torch.cat([Xlock, Xact]))
            _, V = ops.eigh(ops.gram(X, ops.H(X)))
            X.copy_(ops.rot(X, V))
            HX = ops.H(X)
        else:
            HW = ops.H(W)
            Rinv = ops.chol_rinv(ops.gram(W, W))
            W = ops.rot(W, Rinv)
            HW = ops.rot(HW, Rinv)
            if it > 1:
                Q = torch.cat([X, W, P])
                HQ = torch.cat([HX, HW, HP])
            else:
                Q = torch.cat([X, W])
                HQ = torch.cat([HX, HW])
            _, S = ops.eigh(ops.gram(Q, HQ), ops.gram(Q, Q), k=n)
            X.copy_(ops.rot(Q, S))
            HX = ops.rot(HQ, S)
            if it > 1:
                U2, U3 = S[n:2 * n].contiguous(), S[2 * n:3 * n].contiguous()
                Pn = ops.rot(W, U2)
                ops.rot(P, U3, out=Pn, accumulate=True)
                HPn = ops.rot(HW, U2)
                ops.rot(HP, U3, out=HPn, accumulate=True)
                Rinv = ops.chol_rinv(ops.gram(Pn, Pn))
                P = ops.rot(Pn, Rinv)
                HP = ops.rot(HPn, Rinv)
            else:
                P = W.clone()
                HP = HW.clone()
    S = ops.gram(X, HX)
    S = 0.5 * (S + S.conj().T)
    lam, V = ops.eigh(S)
    X.copy_(ops.rot(X, V).to(cdt))
    return lam.cpu().numpy(), niter
