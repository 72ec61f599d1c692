"""Owning wrapper around a ``pw_ctx`` (one basis, one device, one stream).

Device wavefunction blocks are torch tensors of shape (nb, Ngw), contiguous:
row b is band b, i.e. the memory of the reference's column-major
Matrix{ComplexF64}(Ngw, nb) (PWDFT.jl wavefunctions).  Host arrays handed to
the ``*_host`` methods are NumPy (Ngw, nb) arrays in the reference's layout.
"""
import ctypes as C

import numpy as np

from ._lib import (lib, check, pw_grid_desc, pw_tuning, PW_C128, PW_C64, PW_OP_H, PW_ACCUMULATE, PW_GRAPH,
                   PW_PERSISTENT)

TUNING_FIELDS = ("band_chunk_bytes", "plane_bands", "z_columns", "gemm_splits")

_dp = C.POINTER(C.c_double)


def _dptr(a):
    return a.ctypes.data_as(_dp)


def C_void(t):
    return C.c_void_p(t.data_ptr())


def dtype_code(t):
    """Element type code of a torch complex tensor."""
    import torch
    if t.dtype == torch.complex128:
        return PW_C128
    if t.dtype == torch.complex64:
        return PW_C64
    raise TypeError("wavefunctions must be complex128 (FP64 path) or complex64 (mixed precision), got %s" % t.dtype)


class Context:
    """Replaces Ham.pw's FFT plans / index maps plus the operator data
    (V_loc, betaNL, h_ij) of a PWDFT.jl Hamiltonian on one GPU."""

    def __init__(self, Ns, CellVolume, idx_gw2r, Gk2, Nspin=1, device=0, index_base=0):
        self._L = lib()
        self.Ns = tuple(int(n) for n in Ns)
        self.N = int(np.prod(self.Ns))
        self.Nkpt = len(idx_gw2r)
        self.device = device
        self._idx = [np.ascontiguousarray(np.asarray(i, dtype=np.int64)) for i in idx_gw2r]
        self._gk2 = [np.ascontiguousarray(np.asarray(g, dtype=np.float64)) for g in Gk2]
        self.Ngw = [len(i) for i in self._idx]
        ngw = (C.c_int64 * self.Nkpt)(*self.Ngw)
        pidx = (C.POINTER(C.c_int64) * self.Nkpt)(*[a.ctypes.data_as(C.POINTER(C.c_int64)) for a in self._idx])
        pgk2 = (C.POINTER(C.c_double) * self.Nkpt)(*[_dptr(a) for a in self._gk2])
        d = pw_grid_desc()
        d.Ns[:] = list(self.Ns)
        d.Nkpt, d.Nspin, d.index_base, d.CellVolume = self.Nkpt, Nspin, index_base, float(CellVolume)
        d.Ngw = ngw
        d.idx_gw2r = pidx
        d.Gk2 = pgk2
        h = C.c_void_p()
        check(self._L.pw_create(device, C.byref(d), C.byref(h)))
        self.h = h
        self.CellVolume = float(CellVolume)
        self.nbeta = 0
        self._stream = None

    # -------------------------------------------------------------- admin
    def close(self):
        if getattr(self, "h", None):
            self._L.pw_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st):
        check(st, self.h)

    def use_torch_stream(self):
        """Order the library's work on torch's current CUDA stream."""
        import torch
        s = torch.cuda.current_stream(self.device)
        if self._stream is not s:
            self._chk(self._L.pw_set_stream(self.h, C.c_void_p(s.cuda_stream)))
            self._stream = s

    def synchronize(self):
        self._chk(self._L.pw_synchronize(self.h))

    def check_device(self):
        """Raise PWError(PW_ERR_TIMEOUT) if a bounded device wait expired."""
        self._chk(self._L.pw_check_device(self.h))

    def launch_count(self):
        return int(self._L.pw_launch_count(self.h))

    # ------------------------------------------------------------- tuning
    def get_tuning(self):
        """The context's launch parameters (pw_tuning) as a dict; 0 = default."""
        t = pw_tuning()
        self._chk(self._L.pw_get_tuning(self.h, C.byref(t)))
        return {f: int(getattr(t, f)) for f in TUNING_FIELDS}

    def set_tuning(self, **kw):
        """Change some launch parameters (the others keep their values)."""
        cur = self.get_tuning()
        for k, v in kw.items():
            if k not in cur:
                raise KeyError("unknown tuning field %r" % k)
            cur[k] = int(v)
        t = pw_tuning()
        for f in TUNING_FIELDS:
            setattr(t, f, cur[f])
        self._chk(self._L.pw_set_tuning(self.h, C.byref(t)))

    def autotune(self, ik, nb, dtype=PW_C64, cache_path=None):
        """pw_autotune: time candidate launch parameters for op_H on nb bands of
        k-point ik (and the Rayleigh-Ritz products for PW_C64), apply the
        fastest.  Returns (tuning dict, {op_H_default_ms, op_H_tuned_ms,
        rr_default_ms, rr_tuned_ms}); a cache hit reports -1 timings."""
        t = pw_tuning()
        ms = np.zeros(4)
        self.use_torch_stream()
        self._chk(self._L.pw_autotune(self.h, int(ik), int(nb), int(dtype),
                                      None if cache_path is None else str(cache_path).encode(), C.byref(t), _dptr(ms)))
        names = ("op_H_default_ms", "op_H_tuned_ms", "rr_default_ms", "rr_tuned_ms")
        return {f: int(getattr(t, f)) for f in TUNING_FIELDS}, dict(zip(names, ms.tolist()))

    # ------------------------------------------------------------ set-up
    def set_vloc(self, V):
        V = np.asarray(V, dtype=np.float64)
        nspin = 1 if V.ndim == 1 else V.shape[1]
        Vf = np.asfortranarray(V.reshape(self.N, nspin))
        self._chk(self._L.pw_set_vloc(self.h, _dptr(Vf), nspin))

    def set_vloc_device(self, V):
        nspin = 1 if V.dim() == 1 else V.shape[0]
        self.use_torch_stream()
        self._chk(self._L.pw_set_vloc_device(self.h, C.c_void_p(V.data_ptr()), nspin))

    def set_nonlocal(self, ik, betaNL):
        b = np.asfortranarray(np.asarray(betaNL, dtype=np.complex128))
        assert b.shape[0] == self.Ngw[ik]
        self._chk(self._L.pw_set_nonlocal(self.h, ik, b.ctypes.data_as(_dp), b.shape[1]))
        self.nbeta = b.shape[1]

    def set_nonlocal_coef(self, triplets):
        ib = np.array([t[0] for t in triplets], dtype=np.int32)
        jb = np.array([t[1] for t in triplets], dtype=np.int32)
        hv = np.array([t[2] for t in triplets], dtype=np.float64)
        self._chk(self._L.pw_set_nonlocal_coef(self.h, len(triplets), ib.ctypes.data_as(C.POINTER(C.c_int32)),
                                               jb.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(hv)))

    # ----------------------------------------------------- device entry points
    def apply(self, ik, ispin, psi, Hpsi, ops=PW_OP_H):
        """Hpsi (+)= H psi; psi, Hpsi: torch (nb, Ngw) complex, same dtype."""
        assert psi.dtype == Hpsi.dtype and psi.is_contiguous() and Hpsi.is_contiguous()
        nb, ld = psi.shape
        self.use_torch_stream()
        self._chk(self._L.pw_apply(self.h, ik, ispin, dtype_code(psi), C.c_void_p(psi.data_ptr()),
                                   C.c_void_p(Hpsi.data_ptr()), ld, nb, ops))

    def apply_multi(self, iks, ispin, psis, Hpsis, ops=PW_OP_H, graph=False, persistent=False):
        """pw_apply_multi: Hpsis[i] (+)= H(k = iks[i]) psis[i] for every k-point
        in one launch per stage; psis / Hpsis: lists of torch (nb, Ngw)
        blocks of one dtype.  graph=True replays a captured CUDA graph when
        the k-points, blocks and flags repeat."""
        n = len(iks)
        assert n == len(psis) == len(Hpsis) and n > 0
        k = np.ascontiguousarray(np.asarray(iks, dtype=np.int32))
        P = (C.c_void_p * n)(*[p.data_ptr() for p in psis])
        H = (C.c_void_p * n)(*[h.data_ptr() for h in Hpsis])
        ld = np.ascontiguousarray(np.array([p.shape[1] for p in psis], dtype=np.int64))
        nb = np.ascontiguousarray(np.array([p.shape[0] for p in psis], dtype=np.int32))
        for p, h in zip(psis, Hpsis):
            assert p.dtype == psis[0].dtype == h.dtype and p.is_contiguous() and h.is_contiguous()
        self.use_torch_stream()
        self._chk(self._L.pw_apply_multi(self.h, n, k.ctypes.data_as(C.POINTER(C.c_int32)), ispin,
                                         dtype_code(psis[0]), P, H, ld.ctypes.data_as(C.POINTER(C.c_int64)),
                                         nb.ctypes.data_as(C.POINTER(C.c_int32)),
                                         ops | (PW_GRAPH if graph else 0) | (PW_PERSISTENT if persistent else 0)))

    def lobpcg_multi(self, iks, ispin, Xs, tol=1e-5, nitermax=100, nconv=0):
        """pw_lobpcg_multi: the blocks Xs (torch (nb, Ngw) per k-point, one
        dtype) of k-points iks advanced together; returns (evals (nb, nk), niter)."""
        n = len(iks)
        nb = Xs[0].shape[0]
        k = np.ascontiguousarray(np.asarray(iks, dtype=np.int32))
        P = (C.c_void_p * n)(*[x.data_ptr() for x in Xs])
        ld = np.ascontiguousarray(np.array([x.shape[1] for x in Xs], dtype=np.int64))
        ev = np.zeros((n, nb))
        nit = C.c_int(0)
        self.use_torch_stream()
        self._chk(self._L.pw_lobpcg_multi(self.h, n, k.ctypes.data_as(C.POINTER(C.c_int32)), ispin, dtype_code(Xs[0]),
                                          P, ld.ctypes.data_as(C.POINTER(C.c_int64)), nb, float(tol), int(nitermax),
                                          int(nconv), _dptr(ev), C.byref(nit)))
        return ev.T.copy(), nit.value

    def apply_vloc_noalloc(self, ik, ispin, psi, Hpsi, ops):
        """pw_apply_vloc_noalloc: the V_loc (+K) round trip using the library's
        fixed device scratch instead of context-allocated buffers."""
        assert psi.dtype == Hpsi.dtype and psi.is_contiguous() and Hpsi.is_contiguous()
        nb, ld = psi.shape
        self.use_torch_stream()
        self._chk(self._L.pw_apply_vloc_noalloc(self.h, ik, ispin, dtype_code(psi), C.c_void_p(psi.data_ptr()),
                                                C.c_void_p(Hpsi.data_ptr()), ld, nb, ops))

    def kprec(self, ik, x, out):
        nb, ld = x.shape
        self.use_torch_stream()
        self._chk(self._L.pw_kprec(self.h, ik, dtype_code(x), C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
                                   ld, nb))

    def calc_rhoe(self, ik, psi, w, rhoe, accumulate=False):
        """rhoe (torch float64, N) (+)= sum_b w[b] |(N/sqrt(Omega)) G_to_R(psi_b)|^2."""
        nb, ld = psi.shape
        w = np.ascontiguousarray(np.asarray(w, dtype=np.float64))
        assert len(w) == nb
        self.use_torch_stream()
        self._chk(self._L.pw_calc_rhoe(self.h, ik, dtype_code(psi), C.c_void_p(psi.data_ptr()), ld, nb, _dptr(w),
                                       C.c_void_p(rhoe.data_ptr()), int(accumulate)))

    def vloc_vjp(self, ik, psi, w, dV, lam=None, accumulate=False):
        """pw_vloc_vjp: dV (torch float64, N) (+)= the gradient with respect to
        V_loc(r) of sum_b w_b Re<lam_b|V_loc psi_b> (lam None: lam = psi, i.e.
        dE/dV_loc of the band energy with w = wk*Focc)."""
        nb, ld = psi.shape
        w = np.ascontiguousarray(np.asarray(w, dtype=np.float64))
        assert len(w) == nb and (lam is None or (lam.shape == psi.shape and lam.dtype == psi.dtype))
        self.use_torch_stream()
        self._chk(self._L.pw_vloc_vjp(self.h, ik, dtype_code(psi), C.c_void_p(psi.data_ptr()),
                                      None if lam is None else C.c_void_p(lam.data_ptr()), ld, nb, _dptr(w),
                                      C.c_void_p(dV.data_ptr()), int(accumulate)))

    def gram(self, A, B, out, accumulate=False):
        """out (torch complex128, (n, m) row-major = m x n column-major) (+)= A^H B,
        A: (m, K), B: (n, K) band-major blocks."""
        m, K = A.shape
        n = B.shape[0]
        assert out.shape == (n, m) and out.dtype.is_complex and out.element_size() == 16
        self.use_torch_stream()
        self._chk(self._L.pw_gram(self.h, dtype_code(A), K, m, n, C.c_void_p(A.data_ptr()), A.stride(0),
                                  C.c_void_p(B.data_ptr()), B.stride(0), C.c_void_p(out.data_ptr()), m,
                                  int(accumulate)))

    def rotate(self, A, U, out, accumulate=False):
        """out (n, M) (+)= A U: A (k, M) band-major, U complex128 (n, k) row-major
        (= k x n column-major)."""
        k, M = A.shape
        n = U.shape[0]
        assert U.shape[1] == k and out.shape == (n, M)
        self.use_torch_stream()
        self._chk(self._L.pw_rotate(self.h, dtype_code(A), M, n, k, C.c_void_p(A.data_ptr()), A.stride(0),
                                    C.c_void_p(U.data_ptr()), U.stride(0), C.c_void_p(out.data_ptr()), out.stride(0),
                                    int(accumulate)))

    def eigh(self, T, G=None, k=None, vectors=True):
        """Lowest k eigenpairs of (T, G) on the device (FP64): T, G torch
        complex128 (n, n) device tensors holding the column-major matrices
        (i.e. the transposes); both are overwritten.  Returns (lam, S) with
        S a (k, n) tensor (row j = eigenvector j)."""
        import torch
        n = T.shape[0]
        k = n if k is None else k
        lam = torch.empty(k, dtype=torch.float64, device=T.device)
        S = torch.empty((k, n), dtype=torch.complex128, device=T.device) if vectors else None
        self.use_torch_stream()
        self._chk(self._L.pw_eigh(self.h, n, k, C.c_void_p(T.data_ptr()),
                                  C.c_void_p(G.data_ptr()) if G is not None else None, C.c_void_p(lam.data_ptr()),
                                  C.c_void_p(S.data_ptr()) if S is not None else None))
        return lam, S

    def chebyfilt(self, ik, ispin, X, Y, degree, lb, ub):
        """chebyfilt (CheFSI.jl:34-64): Y = p(H) X, the scaled Chebyshev
        filter of `degree` over [lb, ub]; X, Y distinct (nb, Ngw) device
        blocks of one dtype, X unchanged."""
        assert X.dtype == Y.dtype and X.shape == Y.shape and X.is_contiguous() and Y.is_contiguous()
        nb, ld = X.shape
        self.use_torch_stream()
        self._chk(self._L.pw_chebyfilt(self.h, ik, ispin, dtype_code(X), C.c_void_p(X.data_ptr()),
                                       C.c_void_p(Y.data_ptr()), ld, nb, int(degree), float(lb), float(ub)))

    def lanczos_bounds(self, ik, ispin, nlancz, v0):
        """get_ub_lb_lanczos (CheFSI.jl:67-125) from the start vector v0 (a
        complex128 device tensor of Ngw); returns (ub, lb) in the
        reference's order."""
        import torch
        assert v0.dtype == torch.complex128 and v0.is_contiguous()
        lb = C.c_double(0.0)
        ub = C.c_double(0.0)
        self.use_torch_stream()
        self._chk(self._L.pw_lanczos_bounds(self.h, ik, ispin, int(nlancz), C.c_void_p(v0.data_ptr()),
                                            C.byref(lb), C.byref(ub)))
        return ub.value, lb.value

    def ortho_sqrt(self, X):
        """ortho_sqrt!: X (nb, Ngw) device block made orthonormal in place."""
        nb, ld = X.shape
        self.use_torch_stream()
        self._chk(self._L.pw_ortho_sqrt(self.h, dtype_code(X), C.c_void_p(X.data_ptr()), ld, ld, nb))

    def lobpcg(self, ik, ispin, X, tol=1e-5, nitermax=100, nconv=0):
        """diag_LOBPCG!: X (nb, Ngw) device block overwritten; returns (evals, niter)."""
        nb, ld = X.shape
        ev = np.zeros(nb)
        nit = C.c_int(0)
        self.use_torch_stream()
        self._chk(self._L.pw_lobpcg(self.h, ik, ispin, dtype_code(X), C.c_void_p(X.data_ptr()), ld, nb, float(tol),
                                    int(nitermax), int(nconv), _dptr(ev), C.byref(nit)))
        return ev, nit.value

    def davidson(self, ik, ispin, X, tol=1e-8, nitermax=40):
        """diag_davidson_qe!: X (nb, Ngw) device block overwritten with the
        Ritz vectors; returns (evals, niter)."""
        nb, ld = X.shape
        ev = np.zeros(nb)
        nit = C.c_int(0)
        self.use_torch_stream()
        self._chk(self._L.pw_davidson(self.h, ik, ispin, dtype_code(X), C.c_void_p(X.data_ptr()), ld, nb, float(tol),
                                      int(nitermax), _dptr(ev), C.byref(nit)))
        return ev, nit.value

    def set_density_sphere(self, idx_g2r, G2):
        idx = np.ascontiguousarray(np.asarray(idx_g2r, dtype=np.int64))
        g2 = np.ascontiguousarray(np.asarray(G2, dtype=np.float64))
        self._keep_dens = (idx, g2)
        self._chk(self._L.pw_set_density_sphere(self.h, len(idx), idx.ctypes.data_as(C.POINTER(C.c_int64)), _dptr(g2), 0))

    def mix_pulay(self, x, gx, beta, it, mixdim, clamp=True):
        """mix_pulay! on the device (history in the library): x (torch float64,
        N) := the mixed density of iteration it (1 starts a new history),
        clamped at eps() when clamp."""
        self.use_torch_stream()
        self._chk(self._L.pw_mix_pulay(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(gx.data_ptr()), x.numel(),
                                       float(beta), int(it), int(mixdim), int(clamp)))
        return x

    def poisson(self, rho, VH):
        self.use_torch_stream()
        self._chk(self._L.pw_poisson(self.h, C.c_void_p(rho.data_ptr()), C.c_void_p(VH.data_ptr())))

    def update(self, rho, Vps, VH=None, Vxc=None):
        """update!: V_loc := V_ps + V_H[rho] + V_xc[rho] on the device; returns
        (sum V_H rho, sum V_ps rho, sum eps_xc rho)."""
        E3 = np.zeros(3)
        self.use_torch_stream()
        self._chk(self._L.pw_update(self.h, C.c_void_p(rho.data_ptr()), C.c_void_p(Vps.data_ptr()),
                                    C.c_void_p(VH.data_ptr()) if VH is not None else None,
                                    C.c_void_p(Vxc.data_ptr()) if Vxc is not None else None, _dptr(E3)))
        return E3

    def ortho_cholesky(self, psi):
        """ortho_cholesky!: psi (nb, Ngw) device block := psi / chol(psi'psi)."""
        nb, ld = psi.shape
        self.use_torch_stream()
        self._chk(self._L.pw_ortho_cholesky(self.h, dtype_code(psi), C.c_void_p(psi.data_ptr()), ld, ld, nb))

    def chol_rinv(self, C):
        """inv(cholesky(Hermitian(C)).U) on the device: C torch complex128 (n, n)
        holding the column-major matrix (its transpose); returns Rinv in the
        same convention.  C is overwritten."""
        import torch
        n = C.shape[0]
        R = torch.empty_like(C)
        self.use_torch_stream()
        self._chk(self._L.pw_chol_rinv(self.h, n, C_void(C), C_void(R)))
        return R

    def calc_grad(self, ik, ispin, psi, Focc, wk):
        """calc_grad: returns grad (same shape and dtype as psi (nb, Ngw))."""
        import torch
        nb, ld = psi.shape
        g = torch.empty_like(psi)
        f = np.ascontiguousarray(np.asarray(Focc, dtype=np.float64))
        self.use_torch_stream()
        self._chk(self._L.pw_calc_grad(self.h, ik, ispin, dtype_code(psi), C.c_void_p(psi.data_ptr()),
                                       C.c_void_p(g.data_ptr()), ld, nb, _dptr(f), float(wk)))
        return g

    # ---------------------------------------------------------------- forces
    def set_xc(self, xc, G=None):
        """Exchange-correlation of update(): PW_XC_VWN or PW_XC_PBE; G (Ng, 3)
        of the density sphere, in its order (PBE only)."""
        g = None if G is None else np.ascontiguousarray(np.asarray(G, dtype=np.float64))
        self._keep_xc = g
        self._chk(self._L.pw_set_xc(self.h, int(xc), None if g is None else _dptr(g)))

    def build_nonlocal(self, ik, table, positions):
        """pw_build_nonlocal: betaNL of k-point ik evaluated on the device
        from the G+k vectors (set_gkvec first), the column table of
        system.projector_table and the atom positions (3, natoms)."""
        t = {k: np.ascontiguousarray(v) for k, v in table.items()}
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).T)      # column-major 3 x natoms
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        self._chk(self._L.pw_build_nonlocal(self.h, ik, len(t["l"]), ip(t["atom"]), ip(t["l"]), ip(t["m"]),
                                            ip(t["iproj"]), _dptr(t["rc"]), _dptr(t["pref"]), pos.shape[0],
                                            _dptr(pos)))

    def set_symmetry(self, isg, phase):
        """RhoeSymmetrizer tables: isg (nshell, nsym) sphere indices, phase
        (nshell, nsym, 2) cos/sin of G.ft."""
        i = np.ascontiguousarray(np.asarray(isg, dtype=np.int32))
        p = np.ascontiguousarray(np.asarray(phase, dtype=np.float64))
        self._keep_sym = (i, p)
        self._chk(self._L.pw_set_symmetry(self.h, i.shape[0], i.shape[1], i.ctypes.data_as(C.POINTER(C.c_int32)),
                                          _dptr(p)))

    def symmetrize_rhoe(self, rho):
        """symmetrize_rhoe!: the device density rho (N, FP64) in place."""
        self.use_torch_stream()
        self._chk(self._L.pw_symmetrize_rhoe(self.h, C.c_void_p(rho.data_ptr())))

    def set_force_tables(self, VlocG, G):
        """VlocG (Ng, nspecies): eval_Vloc_G per species on the density sphere
        (no 1/Omega); G (Ng, 3) of that sphere, in its order."""
        V = np.ascontiguousarray(np.asarray(VlocG, dtype=np.float64).T)   # column-major Ng x nspecies
        g = np.ascontiguousarray(np.asarray(G, dtype=np.float64))          # column-major 3 x Ng
        self._keep_force = (V, g)
        self._chk(self._L.pw_set_force_tables(self.h, V.shape[0], _dptr(V), _dptr(g)))

    def forces_local(self, rho, positions, species):
        """calc_forces_Ps_loc: rho device (N,), positions (3, natoms), species (natoms,) -> F (3, natoms)."""
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).T)
        sp = np.ascontiguousarray(np.asarray(species, dtype=np.int32))
        F = np.zeros((pos.shape[0], 3))
        self.use_torch_stream()
        self._chk(self._L.pw_forces_local(self.h, C.c_void_p(rho.data_ptr()), pos.shape[0], _dptr(pos),
                                          sp.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(F)))
        return F.T.copy()

    def set_gkvec(self, ik, gk):
        """gk (Ngw, 3): the G+k vectors of k-point ik in the idx_gw2r order."""
        g = np.ascontiguousarray(np.asarray(gk, dtype=np.float64))
        self._chk(self._L.pw_set_gkvec(self.h, ik, _dptr(g)))

    def set_nonlocal_atoms(self, natoms, atom_of_beta):
        a = np.ascontiguousarray(np.asarray(atom_of_beta, dtype=np.int32))
        self._chk(self._L.pw_set_nonlocal_atoms(self.h, int(natoms), a.ctypes.data_as(C.POINTER(C.c_int32))))
        self._force_natoms = int(natoms)

    def forces_nonlocal(self, ik, psi, w):
        """calc_forces_Ps_nloc of one k-point: psi device (nb, Ngw), w (nb,) = wk * Focc -> F (3, natoms)."""
        nb, ld = psi.shape
        ww = np.ascontiguousarray(np.asarray(w, dtype=np.float64))
        F = np.zeros((self._force_natoms, 3))
        self.use_torch_stream()
        self._chk(self._L.pw_forces_nonlocal(self.h, ik, dtype_code(psi), C.c_void_p(psi.data_ptr()), ld, nb,
                                             _dptr(ww), _dptr(F)))
        return F.T.copy()

    def band_energies(self, ik, psi, w):
        """(E_kin, E_Ps_nloc) contributions of k-point ik with weights w = wk*Focc."""
        nb, ld = psi.shape
        w = np.ascontiguousarray(np.asarray(w, dtype=np.float64))
        E2 = np.zeros(2)
        self.use_torch_stream()
        self._chk(self._L.pw_band_energies(self.h, ik, dtype_code(psi), C.c_void_p(psi.data_ptr()), ld, nb, _dptr(w),
                                           _dptr(E2)))
        return E2

    # ---------------------------------------------------------- host drop-ins
    def op_H_host(self, ik, ispin, psi, Hpsi=None, ops=PW_OP_H, dtype=PW_C128):
        """The reference call on host arrays: psi (Ngw, nb) complex128."""
        psi = np.asfortranarray(np.asarray(psi, dtype=np.complex128))
        ld, nb = psi.shape
        if Hpsi is None:
            Hpsi = np.zeros((ld, nb), dtype=np.complex128, order="F")
            ops &= ~PW_ACCUMULATE
        assert Hpsi.flags.f_contiguous and Hpsi.dtype == np.complex128
        self._chk(self._L.pw_op_H_host(self.h, ik, ispin, psi.ctypes.data_as(_dp), Hpsi.ctypes.data_as(_dp), ld, nb,
                                       ops, dtype))
        return Hpsi

    def davidson_host(self, ik, ispin, evc, tol=1e-8, nitermax=40, dtype=PW_C128):
        """diag_davidson_qe!(Ham, evc) on the reference's host array evc
        (Ngw, nb) complex128, overwritten (Fortran order); returns (evals, niter)."""
        assert evc.flags.f_contiguous and evc.dtype == np.complex128
        ld, nb = evc.shape
        ev = np.zeros(nb)
        nit = C.c_int(0)
        self._chk(self._L.pw_davidson_host(self.h, ik, ispin, dtype, evc.ctypes.data_as(_dp), ld, nb, float(tol),
                                           int(nitermax), _dptr(ev), C.byref(nit)))
        return ev, nit.value

    def calc_rhoe_host(self, ik, psi, w, rhoe=None, accumulate=False, dtype=PW_C128):
        psi = np.asfortranarray(np.asarray(psi, dtype=np.complex128))
        ld, nb = psi.shape
        if rhoe is None:
            rhoe = np.zeros(self.N)
            accumulate = False
        w = np.ascontiguousarray(np.asarray(w, dtype=np.float64))
        self._chk(self._L.pw_calc_rhoe_host(self.h, ik, psi.ctypes.data_as(_dp), ld, nb, _dptr(w), _dptr(rhoe),
                                            int(accumulate), dtype))
        return rhoe
