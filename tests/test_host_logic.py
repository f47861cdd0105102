"""Host-side logic of the product path, checked on CPU: the mesh generator and the
2x2 packing.

The product's Clements decomposition and the oracle's are two copies of one seeded
algorithm, so their equality below only shows the copies agree; the check of the
algorithm itself is the reconstruction of U from the mesh and the mesh's shape (the
single-photon known-answer test on the GPU checks it through the simulation too)."""
import numpy as np
import pytest

from bosonsampling_b200 import engine, interferometer
from oracle import circuit, fock, interferometer as ointerf, mpo


@pytest.mark.parametrize("n", [4, 7, 16, 32])
def test_mesh_matches_oracle_and_reconstructs(n):
    U, bs, ph = interferometer.circuit(n, 500 + n)
    U2, bs2, ph2 = ointerf.circuit(n, 500 + n)
    assert np.allclose(U, U2) and bs == bs2 and np.allclose(ph, ph2)
    R = interferometer.mesh_unitary(n, bs, ph)
    assert np.abs(R - U).max() < 1e-12
    assert len(bs) == n * (n - 1) // 2
    assert max(b[0] for b in bs) + 1 == n
    assert all((layer - m) % 2 == 0 for (layer, m, _, _) in bs)   # brick wall, layer 0 even


def test_m8_packing_and_transpose_convention():
    S = np.array([[1 + 2j, 3 - 1j], [0.5j, -2]])
    m = engine._m8(S)
    assert m.tolist() == [1, 2, 3, -1, 0, 0.5, -2, 0]
    # the library builds the tensor of S^T from S; the oracle's update_tensor does the same
    np.testing.assert_allclose(fock.update_tensor(S, 3), fock.bs_tensor(S.T, 3))


def test_workload_table():
    assert circuit.WORKLOADS["precision"] == dict(n=64, eta=0.3, d=5, chi=1024, seed=1003)
    assert circuit.WORKLOADS["plain-scale"]["chi"] == 256
