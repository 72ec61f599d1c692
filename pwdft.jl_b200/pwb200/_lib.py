"""ctypes binding of libpwb200.so (the C ABI declared in include/pwb200.h).

The shared library is built in-tree (``make -C pwdft.jl_b200``) and loaded
from this directory.  There is no fallback: if the library is missing or
cannot be loaded, importing any compute entry point raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpwb200.so")

PW_OK, PW_ERR_ARG, PW_ERR_CUDA, PW_ERR_NOMEM, PW_ERR_NOT_POSDEF, PW_ERR_NAN, PW_ERR_STATE, \
    PW_ERR_UNSUPPORTED, PW_ERR_TIMEOUT = range(9)
PW_C128, PW_C64 = 0, 1
PW_OP_K, PW_OP_VLOC, PW_OP_VNL, PW_OP_H = 1, 2, 4, 7
PW_ACCUMULATE = 0x100
PW_GRAPH = 0x200
PW_PERSISTENT = 0x400
PW_XC_VWN, PW_XC_PBE = 0, 1

STATUS_NAMES = {0: "PW_OK", 1: "PW_ERR_ARG", 2: "PW_ERR_CUDA", 3: "PW_ERR_NOMEM", 4: "PW_ERR_NOT_POSDEF",
                5: "PW_ERR_NAN", 6: "PW_ERR_STATE", 7: "PW_ERR_UNSUPPORTED", 8: "PW_ERR_TIMEOUT"}


class PWError(RuntimeError):
    """A non-zero status from libpwb200 (the reference raises a Julia
    exception in the same situations)."""

    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), msg))
        self.status = status


class pw_grid_desc(C.Structure):
    _fields_ = [("Ns", C.c_int32 * 3), ("Nkpt", C.c_int32), ("Nspin", C.c_int32), ("index_base", C.c_int32),
                ("CellVolume", C.c_double), ("Ngw", C.POINTER(C.c_int64)),
                ("idx_gw2r", C.POINTER(C.POINTER(C.c_int64))), ("Gk2", C.POINTER(C.POINTER(C.c_double)))]


class pw_tuning(C.Structure):
    _fields_ = [("band_chunk_bytes", C.c_int64), ("plane_bands", C.c_int32), ("z_columns", C.c_int32),
                ("gemm_splits", C.c_int32), ("reserved", C.c_int32 * 5)]


_vp, _i, _i64, _d, _u = C.c_void_p, C.c_int, C.c_int64, C.c_double, C.c_uint
_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)

# name -> (restype, argtypes); every symbol of include/pwb200.h
SIGNATURES = {
    "pw_abi_version": (_i, []),
    "pw_create": (_i, [_i, C.POINTER(pw_grid_desc), C.POINTER(_vp)]),
    "pw_destroy": (None, [_vp]),
    "pw_last_error": (C.c_char_p, [_vp]),
    "pw_set_stream": (_i, [_vp, _vp]),
    "pw_synchronize": (_i, [_vp]),
    "pw_launch_count": (_i64, [_vp]),
    "pw_check_device": (_i, [_vp]),
    "pw_device_alloc": (_i, [_vp, C.c_uint64, C.POINTER(_vp)]),
    "pw_device_free": (_i, [_vp, _vp]),
    "pw_copy_to_device": (_i, [_vp, _vp, _vp, C.c_uint64]),
    "pw_copy_to_host": (_i, [_vp, _vp, _vp, C.c_uint64]),
    "pw_get_tuning": (_i, [_vp, C.POINTER(pw_tuning)]),
    "pw_set_tuning": (_i, [_vp, C.POINTER(pw_tuning)]),
    "pw_autotune": (_i, [_vp, _i, _i, _i, C.c_char_p, C.POINTER(pw_tuning), _dp]),
    "pw_set_vloc": (_i, [_vp, _dp, _i]),
    "pw_set_vloc_device": (_i, [_vp, _vp, _i]),
    "pw_set_nonlocal": (_i, [_vp, _i, _dp, _i]),
    "pw_set_nonlocal_coef": (_i, [_vp, _i, _i32p, _i32p, _dp]),
    "pw_apply": (_i, [_vp, _i, _i, _i, _vp, _vp, _i64, _i, _u]),
    "pw_apply_multi": (_i, [_vp, _i, _i32p, _i, _i, C.POINTER(_vp), C.POINTER(_vp), _i64p, _i32p, _u]),
    "pw_lobpcg_multi": (_i, [_vp, _i, _i32p, _i, _i, C.POINTER(_vp), _i64p, _i, _d, _i, _i, _dp, C.POINTER(C.c_int)]),
    "pw_apply_vloc_noalloc": (_i, [_vp, _i, _i, _i, _vp, _vp, _i64, _i, _u]),
    "pw_noalloc_scratch_bytes": (C.c_uint64, []),
    "pw_kprec": (_i, [_vp, _i, _i, _vp, _vp, _i64, _i]),
    "pw_calc_rhoe": (_i, [_vp, _i, _i, _vp, _i64, _i, _dp, _vp, _i]),
    "pw_vloc_vjp": (_i, [_vp, _i, _i, _vp, _vp, _i64, _i, _dp, _vp, _i]),
    "pw_gram": (_i, [_vp, _i, _i64, _i, _i, _vp, _i64, _vp, _i64, _vp, _i64, _i]),
    "pw_rotate": (_i, [_vp, _i, _i64, _i, _i, _vp, _i64, _vp, _i64, _vp, _i64, _i]),
    "pw_eigh": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp]),
    "pw_lobpcg": (_i, [_vp, _i, _i, _i, _vp, _i64, _i, _d, _i, _i, _dp, C.POINTER(C.c_int)]),
    "pw_ortho_sqrt": (_i, [_vp, _i, _vp, _i64, _i64, _i]),
    "pw_lobpcg_host": (_i, [_vp, _i, _i, _i, _dp, _i64, _i, _d, _i, _i, _dp, C.POINTER(C.c_int)]),
    "pw_davidson": (_i, [_vp, _i, _i, _i, _vp, _i64, _i, _d, _i, _dp, C.POINTER(C.c_int)]),
    "pw_davidson_host": (_i, [_vp, _i, _i, _i, _dp, _i64, _i, _d, _i, _dp, C.POINTER(C.c_int)]),
    "pw_chebyfilt": (_i, [_vp, _i, _i, _i, _vp, _vp, _i64, _i, _i, _d, _d]),
    "pw_lanczos_bounds": (_i, [_vp, _i, _i, _i, _vp, _dp, _dp]),
    "pw_set_density_sphere": (_i, [_vp, _i64, _i64p, _dp, _i]),
    "pw_poisson": (_i, [_vp, _vp, _vp]),
    "pw_mix_pulay": (_i, [_vp, _vp, _vp, _i64, _d, _i, _i, _i]),
    "pw_update": (_i, [_vp, _vp, _vp, _vp, _vp, _dp]),
    "pw_band_energies": (_i, [_vp, _i, _i, _vp, _i64, _i, _dp, _dp]),
    "pw_ortho_cholesky": (_i, [_vp, _i, _vp, _i64, _i64, _i]),
    "pw_chol_rinv": (_i, [_vp, _i, _vp, _vp]),
    "pw_calc_grad": (_i, [_vp, _i, _i, _i, _vp, _vp, _i64, _i, _dp, _d]),
    "pw_set_force_tables": (_i, [_vp, _i, _dp, _dp]),
    "pw_set_xc": (_i, [_vp, _i, _dp]),
    "pw_build_nonlocal": (_i, [_vp, _i, _i, _i32p, _i32p, _i32p, _i32p, _dp, _dp, _i, _dp]),
    "pw_set_symmetry": (_i, [_vp, _i, _i, _i32p, _dp]),
    "pw_symmetrize_rhoe": (_i, [_vp, _vp]),
    "pw_forces_local": (_i, [_vp, _vp, _i, _dp, _i32p, _dp]),
    "pw_set_gkvec": (_i, [_vp, _i, _dp]),
    "pw_set_nonlocal_atoms": (_i, [_vp, _i, _i32p]),
    "pw_forces_nonlocal": (_i, [_vp, _i, _i, _vp, _i64, _i, _dp, _dp]),
    "pw_op_H_host": (_i, [_vp, _i, _i, _dp, _dp, _i64, _i, _u, _i]),
    "pw_calc_rhoe_host": (_i, [_vp, _i, _dp, _i64, _i, _dp, _dp, _i, _i]),
    "pw_good_fft_order": (_i, [_i]),
    "pw_gvec_count": (_i, [_i32p, _dp, _d, _i64p]),
    "pw_gvec_build": (_i, [_i32p, _dp, _d, _i64, _dp, _dp, _i64p]),
    "pw_gvecw_build": (_i, [_i64, _dp, _i64p, _dp, _d, _i64p, _i64p, _i64p, _dp]),
}

_lib = None


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libpwb200.so not found at %s: build it with `make -C pwdft.jl_b200`" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status, ctx=None):
    if status != PW_OK:
        msg = lib().pw_last_error(ctx)
        raise PWError(status, msg.decode() if msg else "")
