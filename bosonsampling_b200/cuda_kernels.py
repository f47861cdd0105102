"""Drop-ins for the reference's ``src/cuda_kernels.py`` wrappers.

Same names, argument order and meaning; tensors are torch CUDA tensors instead of
cupy arrays, and the arithmetic is FP64 on sm_100a through libbsmpo.
"""
import ctypes
from cmath import exp
from math import pi, sqrt

import numpy as np

from . import _capi


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("cuda_kernels needs a CUDA device (no CPU path exists)")
    return torch


def Rand_U(d: int, r: float):
    """Random-phase beam-splitter tensor, as ``Rand_U`` (``src/cuda_kernels.py:18-50``).

    Draws the phases from numpy's global RNG in the reference's order (t's phase,
    then r's; for r == 0 the reference uses t = 1 and draws only r's phase) and
    returns ``(U_r, U_i)``: float64 CUDA tensors [d, d, d], U[n, m, l] =
    <l, n+m-l| BS |n, m>.  Evaluated in FP64 with integer powers (no log-domain NaN
    at r = 0, so no host branch is needed).
    """
    torch = _torch()
    if r == 0:
        t = 1.0 + 0j
        rr = r * exp(1j * np.random.rand() * 2 * pi)
    else:
        t = sqrt(1 - r ** 2) * exp(1j * np.random.rand() * 2 * pi)
        rr = r * exp(1j * np.random.rand() * 2 * pi)
    dev = torch.device("cuda", torch.cuda.current_device())
    U_r = torch.empty((d, d, d), dtype=torch.float64, device=dev)
    U_i = torch.empty((d, d, d), dtype=torch.float64, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.check(_capi.lib().bsmpo_unitary_tr(d, t.real, t.imag, rr.real, rr.imag,
                                             ctypes.c_void_p(U_r.data_ptr()),
                                             ctypes.c_void_p(U_i.data_ptr()), stream))
    return U_r, U_i


def _data(x):
    """The array inside the reference's ``Data`` wrapper (``src/mpo_sort.py:6-36``), or x."""
    if isinstance(x, np.ndarray) or hasattr(x, "data_ptr"):
        return x
    return x.data if hasattr(x, "data") else x


def update_MPO(d, charge_c_0, charge_c_1, U_r, U_i, glc_obj, gcr_obj, cl_obj, cr_obj,
               change_charges_C, change_idx_C):
    """One centre-charge sector of the two-site contraction, as ``update_MPO``
    (``src/cuda_kernels.py:101-127``).

    ``glc_obj`` / ``gcr_obj`` are [len_l, len_c] / [len_c, len_r] complex tensors (or
    objects with a ``.data`` tensor), ``cl_obj`` / ``cr_obj`` the [len, 2] charges of
    their rows / columns, and ``change_charges_C`` (2 x changes) with ``change_idx_C``
    the centre charge of each centre index from that index on (the reference's
    change list).  Returns C [len_l, len_r] complex128.  No x8 alignment is needed:
    charges are read per row and column.
    """
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    glc = torch.as_tensor(_data(glc_obj), device=dev).to(torch.complex128).contiguous()
    gcr = torch.as_tensor(_data(gcr_obj), device=dev).to(torch.complex128).contiguous()
    cl = torch.as_tensor(_data(cl_obj), device=dev).to(torch.int32).contiguous()
    cr = torch.as_tensor(_data(cr_obj), device=dev).to(torch.int32).contiguous()
    len_l, len_c = glc.shape
    len_r = gcr.shape[1]
    chg = np.asarray(torch.as_tensor(change_charges_C).cpu()).reshape(2, -1)
    idx = np.asarray(torch.as_tensor(change_idx_C).cpu()).reshape(-1)
    cc = np.full((len_c, 2), d, dtype=np.int32)
    for j in range(len(idx)):
        end = idx[j + 1] if j + 1 < len(idx) else len_c
        cc[idx[j]:end, 0] = chg[0, j]
        cc[idx[j]:end, 1] = chg[1, j]
    cc_t = torch.from_numpy(cc).to(dev)
    U = (torch.as_tensor(U_r, device=dev).to(torch.float64)
         + 1j * torch.as_tensor(U_i, device=dev).to(torch.float64)).to(torch.complex128).contiguous()
    C = torch.empty((len_l, len_r), dtype=torch.complex128, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _capi.check(_capi.lib().bsmpo_contract_sector(
        int(d), int(charge_c_0), int(charge_c_1), ctypes.c_void_p(U.data_ptr()),
        ctypes.c_void_p(glc.data_ptr()), ctypes.c_void_p(gcr.data_ptr()),
        ctypes.c_void_p(cl.data_ptr()), ctypes.c_void_p(cc_t.data_ptr()),
        ctypes.c_void_p(cr.data_ptr()), int(len_l), int(len_c), int(len_r),
        ctypes.c_void_p(C.data_ptr()), stream))
    return C


def update_MPS(d, tau, U_r, U_i, Glc, Gcr, LL, LC, LR, CL, CC, CR, incC):
    """The pure-state (MPS) two-site contraction, as ``update_MPS``
    (``src/cuda_kernels.py:72-90``, kernel ``src/update_kernel.cu:193-769``):
    ``T[l, r] = LL[l] LR[r] sum_c LC[c] Glc[l, c] Gcr[c, r] U[cl - tau, tau - cr, cl - q(c)]``
    over centre entries with ``cl >= q(c) >= cr``.  ``CC`` holds the centre charge of
    every centre index (``incC``, the reference's first-index-per-charge table, is
    accepted for the signature and checked against it).  Returns T [len_l, len_r]
    complex128 (FP64 throughout; the reference computes in FP32)."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())

    def cdev(x, dtype):
        return torch.as_tensor(_data(x), device=dev).to(dtype).contiguous()

    glc, gcr = cdev(Glc, torch.complex128), cdev(Gcr, torch.complex128)
    ll, lc, lr = cdev(LL, torch.float64), cdev(LC, torch.float64), cdev(LR, torch.float64)
    cl, cc, cr = cdev(CL, torch.int32), cdev(CC, torch.int32), cdev(CR, torch.int32)
    len_l, len_c = glc.shape
    len_r = gcr.shape[1]
    inc = np.asarray(torch.as_tensor(incC).cpu()).reshape(-1)
    ccn = cc.cpu().numpy()
    for q, first in enumerate(inc):
        if first >= 0 and first < len_c and ccn[first] != q:
            raise ValueError("incC[%d] = %d does not match the centre charges" % (q, first))
    U = (torch.as_tensor(U_r, device=dev).to(torch.float64)
         + 1j * torch.as_tensor(U_i, device=dev).to(torch.float64)).to(torch.complex128).contiguous()
    T = torch.empty((len_l, len_r), dtype=torch.complex128, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    vp = ctypes.c_void_p
    _capi.check(_capi.lib().bsmpo_contract_mps(
        int(d), int(tau), vp(U.data_ptr()), vp(glc.data_ptr()), vp(gcr.data_ptr()), vp(ll.data_ptr()),
        vp(lc.data_ptr()), vp(lr.data_ptr()), vp(cl.data_ptr()), vp(cc.data_ptr()), vp(cr.data_ptr()),
        int(len_l), int(len_c), int(len_r), vp(T.data_ptr()), stream))
    return T
