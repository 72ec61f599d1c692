"""Plane-wave basis, FFT grid sizes, G-vector index maps and k-point grids.

Oracle (test infrastructure only).  Restates PWDFT.jl:
  fft_support.jl:2-72      allowed / good_fft_order
  PWGrid.jl:62-152         PWGrid constructor (grid size rule, dual=4)
  PWGrid.jl:157-163        mm_to_nn
  PWGrid.jl:199-242        init_gvec (stable sortperm on G2)
  PWGrid.jl:245-275        init_Gshells
  PWGrid.jl:292-322        init_gvecw
  KPoints.jl:121-260       gen_kpoint_grid (identity rotation only + time
                           reversal, i.e. use_symmetry=false)
  gen_lattice.jl:17-28     fcc / cubic lattice vectors (by column)

Index maps are returned 0-based (the reference's are 1-based Int64); the
value of every map entry is the reference's minus one.

Floating point operation order follows the reference loops exactly, so that
G2 -- and therefore the stable sort that orders the G-sphere -- is bit-for-bit
the same: G[a] = (R[a,0]*gi + R[a,1]*gj) + R[a,2]*gk, G2 = (G0^2+G1^2)+G2^2.
"""
import math
import numpy as np


def allowed(nr):
    """fft_support.jl:2-45: True iff nr has only the prime factors 2, 3, 5."""
    mr = nr
    pwr = [0] * 5
    for i, fac in enumerate((2, 3, 5, 7, 11)):
        done = False
        maxpwr = int(round(math.log(float(mr)) / math.log(float(fac)))) + 1
        for _ in range(maxpwr):
            if mr == 1:
                done = True
                break
            if mr % fac == 0:
                mr //= fac
                pwr[i] += 1
        if done:
            break
    if mr != 1:
        return False
    return pwr[3] == 0 and pwr[4] == 0


def good_fft_order(nr):
    """fft_support.jl:48-72."""
    new_nr = nr
    while (not allowed(new_nr)) and new_nr <= 2049:
        new_nr += 1
    if new_nr > 2049:
        raise ValueError("fft_order is too large")
    return new_nr


def gen_lattice_fcc(a):
    """gen_lattice.jl:17-27: columns v1=a/2(-1,0,1), v2=a/2(0,1,1), v3=a/2(-1,1,0)."""
    LL = np.zeros((3, 3))
    LL[:, 0] = 0.5 * a * np.array([-1.0, 0.0, 1.0])
    LL[:, 1] = 0.5 * a * np.array([0.0, 1.0, 1.0])
    LL[:, 2] = 0.5 * a * np.array([-1.0, 1.0, 0.0])
    return LL


def gen_lattice_cubic(a):
    """gen_lattice.jl:3-13."""
    LL = np.zeros((3, 3))
    LL[:, 0] = a * np.array([1.0, 0.0, 0.0])
    LL[:, 1] = a * np.array([0.0, 1.0, 0.0])
    LL[:, 2] = a * np.array([0.0, 0.0, 1.0])
    return LL


def recvecs_of(LatVecs):
    """PWGrid.jl:75: RecVecs = 2*pi*inv(LatVecs')  (rows are b-vectors)."""
    return 2 * np.pi * np.linalg.inv(np.ascontiguousarray(LatVecs.T))


def grid_size(LatVecs, ecutrho):
    """PWGrid.jl:79-92: Ns_i = good_fft_order(2*round(sqrt(ecutrho/2)*|a_i|/pi)+1)."""
    Ns = []
    for i in range(3):
        L = float(np.linalg.norm(LatVecs[:, i]))
        n = 2 * int(round(math.sqrt(ecutrho / 2) * L / math.pi)) + 1
        Ns.append(good_fft_order(n))
    return tuple(Ns)


def mm_to_nn(n):
    """PWGrid.jl:157-163 vectorised over 0..n-1."""
    m = np.arange(n)
    return np.where(m > n / 2, m - n, m)


class GVectors:
    pass


class GVectorsW:
    pass


class KPoints:
    def __init__(self, Nkpt, mesh, k, wk, RecVecs):
        self.Nkpt = Nkpt
        self.mesh = mesh
        self.k = k            # (3, Nkpt) Cartesian, 1/bohr
        self.wk = wk          # (Nkpt,), sums to 1
        self.RecVecs = RecVecs


def gamma_kpoints(RecVecs):
    """PWGrid.jl:137-139: single Gamma point, weight 1."""
    return KPoints(1, (1, 1, 1), np.zeros((3, 1)), np.array([1.0]), RecVecs)


def init_gvec(Ns, RecVecs, ecutrho):
    """PWGrid.jl:199-242 (with calc_Ng folded in)."""
    N1, N2, N3 = Ns
    nn1, nn2, nn3 = mm_to_nn(N1), mm_to_nn(N2), mm_to_nn(N3)
    # loop order k (outer), j, i (inner)  ->  ip = i + N1*(j + N2*k)
    gk, gj, gi = np.meshgrid(nn3.astype(np.float64), nn2.astype(np.float64),
                             nn1.astype(np.float64), indexing="ij")
    gi = gi.ravel(); gj = gj.ravel(); gk = gk.ravel()
    R = RecVecs
    G0 = R[0, 0] * gi + R[0, 1] * gj + R[0, 2] * gk
    G1 = R[1, 0] * gi + R[1, 1] * gj + R[1, 2] * gk
    G2c = R[2, 0] * gi + R[2, 1] * gj + R[2, 2] * gk
    G2 = G0 * G0 + G1 * G1 + G2c * G2c
    sel = np.nonzero(0.5 * G2 <= ecutrho)[0]
    order = np.argsort(G2[sel], kind="stable")
    idx = sel[order]
    gv = GVectors()
    gv.Ng = len(idx)
    gv.G = np.stack([G0[idx], G1[idx], G2c[idx]])
    gv.G2 = G2[idx]
    gv.idx_g2r = idx.astype(np.int64)
    gv.miller = np.stack([gi[idx], gj[idx], gk[idx]]).astype(np.int64)
    gv.G2_shells, gv.idx_g2shells = init_Gshells(gv.G2)
    return gv


def init_Gshells(G2_sorted):
    """PWGrid.jl:245-275 (idx_g2shells returned 0-based)."""
    eps8 = 1e-8
    new_shell = np.empty(len(G2_sorted), dtype=bool)
    new_shell[0] = False
    new_shell[1:] = G2_sorted[1:] > (G2_sorted[:-1] + eps8)
    idx = np.cumsum(new_shell).astype(np.int64)
    shells = np.concatenate([[G2_sorted[0]], G2_sorted[1:][new_shell[1:]]])
    return shells, idx


def init_gvecw(ecutwfc, gvec, kpoints):
    """PWGrid.jl:292-322."""
    G = gvec.G
    gw = GVectorsW()
    gw.idx_gw2g, gw.idx_gw2r, gw.Ngw = [], [], []
    for ik in range(kpoints.Nkpt):
        k = kpoints.k[:, ik]
        a = G[0] + k[0]
        b = G[1] + k[1]
        c = G[2] + k[2]
        Gk2 = a * a + b * b + c * c
        i2g = np.nonzero(0.5 * Gk2 <= ecutwfc)[0].astype(np.int64)
        gw.idx_gw2g.append(i2g)
        gw.idx_gw2r.append(gvec.idx_g2r[i2g])
        gw.Ngw.append(len(i2g))
    gw.Ngwx = max(gw.Ngw)
    gw.kpoints = kpoints
    return gw


class PWGrid:
    """PWGrid.jl:62-152 for dual = 4 (no smooth grid)."""

    def __init__(self, ecutwfc, LatVecs, kpoints=None, Ns=None):
        self.ecutwfc = float(ecutwfc)
        self.ecutrho = 4.0 * self.ecutwfc
        self.LatVecs = np.array(LatVecs, dtype=np.float64)
        self.RecVecs = recvecs_of(self.LatVecs)
        self.CellVolume = abs(np.linalg.det(self.LatVecs))
        self.Ns = tuple(Ns) if Ns is not None else grid_size(self.LatVecs, self.ecutrho)
        self.Npoints = int(np.prod(self.Ns))
        self.gvec = init_gvec(self.Ns, self.RecVecs, self.ecutrho)
        if kpoints is None:
            kpoints = gamma_kpoints(self.RecVecs)
        self.gvecw = init_gvecw(self.ecutwfc, self.gvec, kpoints)

    @property
    def kpoints(self):
        return self.gvecw.kpoints

    def Gk2(self, ik):
        """|G+k|^2 over the wavefunction sphere of k-point ik (op_K.jl:67-72)."""
        idx = self.gvecw.idx_gw2g[ik]
        k = self.kpoints.k[:, ik]
        G = self.gvec.G
        return (G[0, idx] + k[0]) ** 2 + (G[1, idx] + k[1]) ** 2 + (G[2, idx] + k[2]) ** 2


def gen_kpoint_grid(LatVecs, nk, shift=(0, 0, 0), time_reversal=True):
    """KPoints.jl:121-260 with the identity as the only rotation (no
    symmetry reduction beyond k ~ -k)."""
    nk1, nk2, nk3 = nk
    k1, k2, k3 = shift
    SMALL = 1.0e-5
    nkr = nk1 * nk2 * nk3
    xkg = np.zeros((3, nkr))
    for i in range(nk1):
        for j in range(nk2):
            for k in range(nk3):
                ik = k + j * nk3 + i * nk2 * nk3
                xkg[0, ik] = i / nk1 + k1 / 2.0 / nk1
                xkg[1, ik] = j / nk2 + k2 / 2.0 / nk2
                xkg[2, ik] = k / nk3 + k3 / 2.0 / nk3
    equiv = np.arange(nkr)
    wkk = np.zeros(nkr)

    def locate(x):
        xx = x[0] * nk1 - 0.5 * k1
        yy = x[1] * nk2 - 0.5 * k2
        zz = x[2] * nk3 - 0.5 * k3
        ok = (abs(xx - round(xx)) <= SMALL and abs(yy - round(yy)) <= SMALL
              and abs(zz - round(zz)) <= SMALL)
        if not ok:
            return None
        i = round(x[0] * nk1 - 0.5 * k1 + 2 * nk1) % nk1
        j = round(x[1] * nk2 - 0.5 * k2 + 2 * nk2) % nk2
        k = round(x[2] * nk3 - 0.5 * k3 + 2 * nk3) % nk3
        return k + j * nk3 + i * nk2 * nk3

    for ik in range(nkr):
        if equiv[ik] != ik:
            continue
        wkk[ik] = 1.0
        xkr = xkg[:, ik] - np.round(xkg[:, ik])
        cands = [xkr]
        if time_reversal:
            cands.append(-xkr)
        for x in cands:
            n = locate(x)
            if n is None:
                continue
            if n > ik and equiv[n] == n:
                equiv[n] = ik
                wkk[ik] += 1.0
            elif equiv[n] != ik or n < ik:
                raise RuntimeError("gen_kpoint_grid: inconsistent equivalence")
    irr = [ik for ik in range(nkr) if equiv[ik] == ik]
    wk = np.array([wkk[ik] for ik in irr])
    xk = np.stack([xkg[:, ik] - np.round(xkg[:, ik]) for ik in irr], axis=1)
    RecVecs = recvecs_of(LatVecs)
    wk = wk / wk.sum()
    xk = RecVecs @ xk
    return KPoints(len(irr), tuple(nk), xk, wk, RecVecs)
