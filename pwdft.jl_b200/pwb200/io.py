"""Wavefunction files in the reference's format.

  write_psiks   KS_solve_SCF_potmix.jl:301-307, KS_solve_DCM.jl:295-300 (savewfc):
                one file WFC_ikspin_<ikspin>.data per (k-point, spin), ikspin =
                ik + (ispin - 1) Nkpt counted from 1, holding the raw
                little-endian ComplexF64 values of psiks[ikspin], Ngw x Nstates
                column-major (Julia's write of a Matrix{ComplexF64})
  read_psiks    read_psiks.jl:1-21: the same files back, one block per ikspin

A device block here is a torch (Nstates, Ngw) tensor, whose row-major bytes
are the column-major Ngw x Nstates matrix, so a complex128 block is written
and read without reordering; complex64 blocks are widened on the device
first (and narrowed after reading when dtype is complex64).
"""
import os

import numpy as np


def wfc_path(ikspin, directory="."):
    """File of block ikspin (0-based here; the name counts from 1)."""
    return os.path.join(directory, "WFC_ikspin_%d.data" % (ikspin + 1))


def write_psiks(psiks, directory="."):
    """Writes every block of psiks (device (Nstates, Ngw) tensors or host
    (Ngw, Nstates) complex arrays) to WFC_ikspin_<n>.data."""
    for i, p in enumerate(psiks):
        if hasattr(p, "detach"):
            import torch
            a = p.detach().to(torch.complex128).contiguous().cpu().numpy()     # (Nstates, Ngw) = column-major
        else:
            a = np.asarray(p, dtype=np.complex128).T                          # host (Ngw, Nstates)
        np.ascontiguousarray(a).astype("<c16", copy=False).tofile(wfc_path(i, directory))


def read_psiks(Ngw, Nstates, Nspin=1, directory=".", device=None, dtype=None):
    """Reads Nspin * len(Ngw) blocks.  device=None returns host (Ngw, Nstates)
    complex128 arrays; otherwise torch (Nstates, Ngw) tensors on device, of
    dtype (complex128 by default)."""
    Nkpt = len(Ngw)
    out = []
    for ispin in range(Nspin):
        for ik in range(Nkpt):
            ikspin = ik + ispin * Nkpt
            path = wfc_path(ikspin, directory)
            n = int(Ngw[ik]) * int(Nstates)
            a = np.fromfile(path, dtype="<c16")
            if a.size != n:
                raise ValueError("%s holds %d values, expected Ngw %d x Nstates %d" % (path, a.size, Ngw[ik], Nstates))
            a = a.reshape(Nstates, int(Ngw[ik]))
            if device is None:
                out.append(np.ascontiguousarray(a.T))
            else:
                import torch
                t = torch.from_numpy(a).to(device)
                out.append((t if dtype is None else t.to(dtype)).contiguous())
    return out
