"""The tensor-core contraction primitive (tcgen05, 3 x TF32 split products) and the
TF32X3 precision mode against FP64.

Tolerances (written here): the GEMM within 2e-6 of max|A| max|B| K (a few times the
2^-21 split error); the TF32X3 circuit within 3e-4 of the trace in every marginal of
the FP64 plain path (its measured error is ~1e-4: see the test).
"""
import ctypes
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from bosonsampling_b200 import _capi, engine, interferometer  # noqa: E402
from oracle import circuit  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    torch.cuda.set_device(0)


def _cplx(rng, *shape):
    return torch.from_numpy(rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).cuda()


@pytest.mark.parametrize("M,N,K,opA", [(128, 64, 8, 0), (200, 130, 77, 0), (37, 300, 513, 0),
                                       (96, 150, 260, 1), (5, 3, 2, 1), (300, 64, 1000, 1)])
def test_zgemm_tf32x3_matches_fp64(M, N, K, opA):
    rng = np.random.default_rng(M * 7 + N + K)
    A = _cplx(rng, K, M) if opA else _cplx(rng, M, K)
    B = _cplx(rng, K, N)
    C = torch.full((M, N), float("nan"), dtype=torch.complex128, device="cuda")
    L = _capi.lib()
    lda = M if opA else K
    rc = L.bsmpo_zgemm_tf32x3(M, N, K, ctypes.c_void_p(A.data_ptr()), lda, opA, ctypes.c_void_p(B.data_ptr()),
                              N, ctypes.c_void_p(C.data_ptr()), N,
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.bsmpo_last_error(None)
    ref = (A.conj().T if opA else A) @ B
    err = (C - ref).abs().max().item()
    assert err <= 2e-6 * A.abs().max().item() * B.abs().max().item() * K, err


def test_tf32x3_circuit_error_bound():
    """Workload 2 (N=32, chi=256, 496 updates) in TF32X3 mode against the FP64 fixture.

    The split-TF32 contraction with FP32 accumulation does not reach the 1e-6 target on
    this circuit (measured ~1e-4 of the trace); the test pins that bound, 3e-4, so a
    regression of the tensor-core path shows."""
    fx = np.load(os.path.join(GOLDEN, "oracle_plain_scale.npz"))
    w = circuit.WORKLOADS["plain-scale"]
    U, bs, ph = interferometer.circuit(w["n"], w["seed"])
    with engine.MPOSimulator(w["n"], w["d"], w["chi"]) as sim:
        sim.set_precision("tf32x3")
        sim.init_single_photons(range(0, w["n"], 2), w["eta"])
        sim.run_mesh([b[1] for b in bs], [b[2] for b in bs], [b[3] for b in bs])
        sim.apply_phases(ph)
        tr, P = sim.observables()
        routes = sim.svd_routes()
    tr_o = complex(fx["trace"][0])
    err = np.abs(P - fx["marginals"]).max() / abs(tr_o)
    assert err <= 3e-4, err
    assert routes[1] > 0   # the Gram route (with its tensor-core contractions) ran
