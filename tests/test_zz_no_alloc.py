"""bsmpo_trace_noalloc: the allocation-free trace for callers that cannot allocate
device memory (e.g. under a framework whose allocator owns the whole device).

Checked through the C ABI against the allocating entry point (bsmpo_observables)
on the same state, on two calls in a row (the second call reuses the library's
fixed scratch array, so stale contents would show up there).  This file is collected
last on purpose.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from bosonsampling_b200 import _capi, engine, interferometer  # noqa: E402

TOL = 1e-10


def _state(n, d, chi, seed, nbs):
    U, bs, ph = interferometer.circuit(n, seed)
    sim = engine.MPOSimulator(n, d, chi)
    sim.init_single_photons(range(0, n, 2), 0.5)
    for (l, m, th, p) in bs[:nbs]:
        sim.bs_update(m, interferometer.t_block(th, p))
    return sim


@pytest.mark.parametrize("n,d,chi,seed,nbs", [(8, 3, 32, 3, 20), (12, 4, 96, 9, 50)])
def test_trace_noalloc_matches_allocating_entry_point(n, d, chi, seed, nbs):
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    L = _capi.lib()
    sim = _state(n, d, chi, seed, nbs)
    ref, _ = sim.observables(marginals=False)
    g, lam, chg = sim.store()
    sim.close()
    _check_two_calls(L, n, d, chi, g, lam, chg, ref)


def _check_two_calls(L, n, d, chi, g, lam, chg, ref):
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    free_after = []
    for call in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = L.bsmpo_trace_noalloc(n, d, chi, ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(lam.data_ptr()),
                                   ctypes.c_void_p(chg.data_ptr()), ctypes.c_void_p(out.data_ptr()), stream)
        assert rc == 0, L.bsmpo_last_error(None)
        torch.cuda.synchronize()
        free_after.append(torch.cuda.mem_get_info()[0])
        tr = complex(out[0].item(), out[1].item())
        assert abs(tr - ref) <= TOL * abs(ref), (call, tr, ref)
    # the second call takes no device memory (the first may: it loads the library's code)
    assert free_after[1] == free_after[0], free_after


def test_trace_noalloc_at_the_largest_chi():
    """chi = BSMPO_NOALLOC_MAX_CHI itself (4096): a three-mode product state padded to
    that bond dimension, against the allocating entry point."""
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    L = _capi.lib()
    n, d, chi = 3, 3, 4096
    with engine.MPOSimulator(n, d, chi) as sim:
        sim.init_single_photons([0, 2], 0.5, canonicalize=False)
        ref, _ = sim.observables(marginals=False)
        g, lam, chg = sim.store()
    _check_two_calls(L, n, d, chi, g, lam, chg, ref)


def test_trace_noalloc_rejects_too_large_chi():
    L = _capi.lib()
    big = 4097
    rc = L.bsmpo_trace_noalloc(4, 3, big, ctypes.c_void_p(1), ctypes.c_void_p(1), ctypes.c_void_p(1),
                               ctypes.c_void_p(1), None)
    assert rc == -1
    assert b"exceeds the allocation-free limit" in L.bsmpo_last_error(None)
