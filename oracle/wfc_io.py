"""Wavefunction files: read_psiks.jl:1-21 and the savewfc writer of
KS_solve_DCM.jl:295-300 (Julia's write/read! of a Matrix{ComplexF64}:
raw little-endian values, column-major, WFC_ikspin_<ikspin>.data with
ikspin counted from 1).

Oracle (test infrastructure only).
"""
import os

import numpy as np


def write_wfc(psiks, directory):
    for i, psi in enumerate(psiks):
        with open(os.path.join(directory, "WFC_ikspin_" + str(i + 1) + ".data"), "wb") as f:
            f.write(np.asfortranarray(psi, dtype=np.complex128).tobytes(order="F"))


def read_wfc(Ngw, Nstates, directory, Nspin=1):
    out = []
    for ispin in range(Nspin):
        for ik in range(len(Ngw)):
            ikspin = ik + ispin * len(Ngw) + 1
            with open(os.path.join(directory, "WFC_ikspin_" + str(ikspin) + ".data"), "rb") as f:
                raw = f.read()
            out.append(np.frombuffer(raw, dtype="<c16").reshape((Ngw[ik], Nstates), order="F").copy())
    return out
