"""GTH pseudopotentials and real spherical harmonics.

Oracle (test infrastructure only).  Restates PWDFT.jl:
  PsPot_GTH.jl:43-118    file parser
  PsPot_GTH.jl:164-217   eval_Vloc_G (G=0 term with the QE/PspCore constant)
  PsPot_GTH.jl:338-391   eval_proj_G
  Ylm_real.jl:5-107      Ylm_real (QE convention, l <= 3)
"""
import math
import numpy as np

ZATOMS = {"Pt": 78, "H": 1, "He": 2, "Li": 3, "C": 6, "N": 7, "O": 8, "Na": 11, "Mg": 12,
          "Al": 13, "Si": 14, "P": 15, "S": 16, "Cl": 17, "Ga": 31, "Ge": 32}


class PsPot_GTH:
    """PsPot_GTH.jl:8-20 / 43-118."""

    def __init__(self, filename):
        self.pspfile = filename
        with open(filename) as f:
            lines = [ln for ln in f.read().splitlines()]
        it = iter(lines)
        self.atsymb = next(it).split()[0]
        n = [int(x) for x in next(it).split()[:4]]
        self.zval = sum(n)
        l = next(it).split()
        self.rlocal = float(l[0])
        n_c_local = int(l[1])
        self.c = np.zeros(4)
        l = next(it).split()
        for i in range(n_c_local):
            self.c[i] = float(l[i])
        self.lmax = int(next(it).split()[0]) - 1
        self.rc = np.zeros(4)
        self.Nproj_l = np.zeros(4, dtype=np.int64)
        self.h = np.zeros((4, 3, 3))
        for i in range(self.lmax + 1):
            l = next(it).split()
            self.rc[i] = float(l[0])
            self.Nproj_l[i] = int(float(l[1]))
            for ii in range(self.Nproj_l[i]):
                l = next(it).split()
                for iread, iii in enumerate(range(ii, self.Nproj_l[i])):
                    self.h[i, ii, iii] = float(l[iread])
        for k in range(4):
            for i in range(3):
                for j in range(i + 1, 3):
                    self.h[k, j, i] = self.h[k, i, j]


def eval_Vloc_G(psp, G2):
    """PsPot_GTH.jl:164-189, vectorised over G2."""
    G2 = np.asarray(G2, dtype=np.float64)
    rloc, zval = psp.rlocal, psp.zval
    c1, c2, c3, c4 = psp.c
    pre1 = -4 * np.pi * zval
    pre2 = math.sqrt(8 * np.pi ** 3) * rloc ** 3
    G2l = np.sqrt(G2)
    Gr = G2l * rloc
    expGr2 = np.exp(-0.5 * Gr ** 2)
    big = np.sqrt(G2l) > 1.0e-8
    with np.errstate(divide="ignore", invalid="ignore"):
        Vg = pre1 / G2 * expGr2 + pre2 * expGr2 * (
            c1 + c2 * (3.0 - Gr ** 2) + c3 * (15.0 - 10.0 * Gr ** 2 + Gr ** 4)
            + c4 * (105.0 - 105.0 * Gr ** 2 + 21.0 * Gr ** 4 - Gr ** 6))
    V0 = 2 * np.pi * zval * rloc ** 2 + (2 * np.pi) ** 1.5 * rloc ** 3 * (
        c1 + 3.0 * c2 + 15.0 * c3 + 105.0 * c4)
    return np.where(big, Vg, V0)


def eval_proj_G(psp, l, iproj, Gm, CellVolume):
    """PsPot_GTH.jl:338-391 (iproj is 1-based as in the reference)."""
    Gm = np.asarray(Gm, dtype=np.float64)
    rrl = psp.rc[l]
    Gr2 = (Gm * rrl) ** 2
    e = np.exp(-0.5 * Gr2)
    if l == 0:
        if iproj == 1:
            V = e
        elif iproj == 2:
            V = 2.0 / math.sqrt(15.0) * e * (3.0 - Gr2)
        else:
            V = (4.0 / 3.0) / math.sqrt(105.0) * e * (15.0 - 10.0 * Gr2 + Gr2 ** 2)
    elif l == 1:
        if iproj == 1:
            V = (1.0 / math.sqrt(3.0)) * e * Gm
        elif iproj == 2:
            V = (2.0 / math.sqrt(105.0)) * e * Gm * (5.0 - Gr2)
        else:
            V = (4.0 / 3.0) / math.sqrt(1155.0) * e * Gm * (35.0 - 14.0 * Gr2 + Gr2 ** 2)
    elif l == 2:
        if iproj == 1:
            V = (1.0 / math.sqrt(15.0)) * e * Gm ** 2
        else:
            V = (2.0 / 3.0) / math.sqrt(105.0) * e * Gm ** 2 * (7.0 - Gr2)
    else:
        V = Gm ** 3 * e / math.sqrt(105.0)
    pre = 4.0 * np.pi ** (5.0 / 4.0) * math.sqrt(2.0 ** (l + 1) * rrl ** (2 * l + 3) / CellVolume)
    return pre * V


def Ylm_real(l, m, R):
    """Ylm_real.jl:5-107, vectorised: R has shape (3, n)."""
    SMALL = 1.0e-9
    x, y, z = R[0], R[1], R[2]
    Rmod = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        cost = np.where(Rmod < SMALL, 0.0, z / Rmod)
        ratio = y / x
        phi = np.where(x > SMALL, np.arctan(ratio),
                       np.where(x < -SMALL, np.arctan(ratio) + np.pi,
                                np.where(y >= 0, np.pi / 2, -np.pi / 2)))
    sint = np.sqrt(np.maximum(0.0, 1.0 - cost ** 2))
    if l == 0:
        return np.full(x.shape, 0.5 * math.sqrt(1.0 / np.pi))
    if l == 1:
        c = 0.5 * math.sqrt(3.0 / np.pi)
        return {-1: c * sint * np.sin(phi), 0: c * cost, 1: c * sint * np.cos(phi)}[m]
    if l == 2:
        if m == -2:
            return math.sqrt(15.0 / 16.0 / np.pi) * sint ** 2 * np.sin(2.0 * phi)
        if m == -1:
            return math.sqrt(15.0 / 4.0 / np.pi) * cost * sint * np.sin(phi)
        if m == 0:
            return 0.25 * math.sqrt(5.0 / np.pi) * (3.0 * cost ** 2 - 1.0)
        if m == 1:
            return math.sqrt(15.0 / 4.0 / np.pi) * cost * sint * np.cos(phi)
        return math.sqrt(15.0 / 16.0 / np.pi) * sint ** 2 * np.cos(2.0 * phi)
    if m == -3:
        return 0.25 * math.sqrt(35.0 / 2.0 / np.pi) * sint ** 3 * np.sin(3.0 * phi)
    if m == -2:
        return 0.25 * math.sqrt(105.0 / np.pi) * sint ** 2 * cost * np.sin(2.0 * phi)
    if m == -1:
        return 0.25 * math.sqrt(21.0 / 2.0 / np.pi) * sint * (5.0 * cost ** 2 - 1.0) * np.sin(phi)
    if m == 0:
        return 0.25 * math.sqrt(7.0 / np.pi) * (5.0 * cost ** 3 - 3.0 * cost)
    if m == 1:
        return 0.25 * math.sqrt(21.0 / 2.0 / np.pi) * sint * (5.0 * cost ** 2 - 1.0) * np.cos(phi)
    if m == 2:
        return 0.25 * math.sqrt(105.0 / np.pi) * sint ** 2 * cost * np.cos(2.0 * phi)
    return 0.25 * math.sqrt(35.0 / 2.0 / np.pi) * sint ** 3 * np.cos(3.0 * phi)
