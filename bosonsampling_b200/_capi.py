"""ctypes binding of libbsmpo.so (declared in include/bsmpo.h).

The library is loaded from this package directory.  There is no fallback: if the
shared library is missing, ``lib()`` raises, so nothing silently runs elsewhere.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbsmpo.so")

_c_int = ctypes.c_int
_c_double = ctypes.c_double
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)

# name -> (restype, argtypes); mirrors include/bsmpo.h
SIGNATURES = {
    "bsmpo_version": (ctypes.c_char_p, []),
    "bsmpo_last_error": (ctypes.c_char_p, [_vp]),
    "bsmpo_unitary": (_c_int, [_c_int, _dp, _vp, _vp]),
    "bsmpo_bs_angle_grad": (_c_int, [_c_int, _c_int, _dp, _dp, _vp, _vp, _vp]),
    "bsmpo_unitary_tr": (_c_int, [_c_int, _c_double, _c_double, _c_double, _c_double, _vp, _vp, _vp]),
    "bsmpo_contract_sector": (_c_int, [_c_int, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp, _vp,
                                       _c_int, _c_int, _c_int, _vp, _vp]),
    "bsmpo_contract_mps": (_c_int, [_c_int, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                    _c_int, _c_int, _c_int, _vp, _vp]),
    "bsmpo_zgemm_tf32x3": (_c_int, [_c_int, _c_int, _c_int, _vp, _c_int, _c_int, _vp, _c_int, _vp, _c_int,
                                    _vp]),
    "bsmpo_create": (_c_int, [_c_int, _c_int, _c_int, _c_int, ctypes.POINTER(_vp)]),
    "bsmpo_destroy": (_c_int, [_vp]),
    "bsmpo_set_stream": (_c_int, [_vp, _vp]),
    "bsmpo_set_cutoff": (_c_int, [_vp, _c_double]),
    "bsmpo_set_precision": (_c_int, [_vp, _c_int]),
    "bsmpo_set_workers": (_c_int, [_vp, _c_int]),
    "bsmpo_load_state": (_c_int, [_vp, _vp, _vp, _vp]),
    "bsmpo_store_state": (_c_int, [_vp, _vp, _vp, _vp]),
    "bsmpo_get_site": (_c_int, [_vp, _c_int, _vp]),
    "bsmpo_put_site": (_c_int, [_vp, _c_int, _vp]),
    "bsmpo_get_bond": (_c_int, [_vp, _c_int, _vp, _vp]),
    "bsmpo_put_bond": (_c_int, [_vp, _c_int, _vp, _vp]),
    "bsmpo_init_product": (_c_int, [_vp, _dp, _c_int]),
    "bsmpo_canonicalize": (_c_int, [_vp]),
    "bsmpo_bs_update": (_c_int, [_vp, _c_int, _dp]),
    "bsmpo_bs_update_tensor": (_c_int, [_vp, _c_int, _vp]),
    "bsmpo_run_mesh": (_c_int, [_vp, _c_int, _ip, _dp, _dp]),
    "bsmpo_run_mesh_host": (_c_int, [_vp, _c_int, _ip, _dp, _dp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "bsmpo_mesh_truncation": (_c_int, [_vp, _dp, _c_int]),
    "bsmpo_apply_phases": (_c_int, [_vp, _dp]),
    "bsmpo_observables": (_c_int, [_vp, _dp, _dp]),
    "bsmpo_last_update_info": (_c_int, [_vp, _ip, _ip, _ip, _ip, _dp, _c_int, _ip, _dp]),
    "bsmpo_last_update_work": (_c_int, [_vp, _dp, _dp, _dp]),
    "bsmpo_bond_dims": (_c_int, [_vp, _ip]),
    "bsmpo_kernel_launches": (ctypes.c_int64, [_vp]),
    "bsmpo_svd_routes": (_c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "bsmpo_workspace_stats": (_c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "bsmpo_stage_times": (_c_int, [_vp, _dp, _c_int]),
    "bsmpo_set_timing": (_c_int, [_vp, _c_int]),
    "bsmpo_jacobi_timing": (_c_int, [_vp, _dp, _dp, ctypes.POINTER(ctypes.c_int64)]),
    "bsmpo_tridiag_timing": (_c_int, [_vp, _dp, _dp, _dp, ctypes.POINTER(ctypes.c_int64)]),
    "bsmpo_trace_noalloc": (_c_int, [_c_int, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp]),
}

_lib = None


class BsmpoError(RuntimeError):
    """A libbsmpo call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__("libbsmpo error %d: %s" % (code, msg))
        self.code = code


def lib():
    """Load libbsmpo.so (once); raises if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libbsmpo.so not found at %s; build it with `python -m bosonsampling_b200.build`"
                % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc, handle=None):
    if rc != 0:
        msg = lib().bsmpo_last_error(handle)
        raise BsmpoError(rc, msg.decode() if msg else "")


def dptr(arr):
    """ctypes double* of a contiguous float64 numpy array."""
    return arr.ctypes.data_as(_dp)


def iptr(arr):
    return arr.ctypes.data_as(_ip)
