"""Host-side logic of the product path, checked on CPU: state builder, mesh
generator and the 2x2 packing, against the oracle's independent versions."""
import numpy as np
import pytest

from bosonsampling_b200 import engine, interferometer
from oracle import circuit, fock, interferometer as ointerf, mpo


@pytest.mark.parametrize("n,d,chi", [(6, 3, 16), (16, 4, 64), (9, 5, 32)])
def test_product_state_matches_oracle(n, d, chi):
    rhos = engine.lossy_single_photon_rhos(n, range(0, n, 2), 0.4, d)
    g, l, c = engine.product_state(n, rhos, d, chi)
    st = mpo.product_state(n, [mpo.single_photon_rho(d, 0.4) if i % 2 == 0 else mpo.vacuum_rho(d)
                               for i in range(n)], d, chi)
    np.testing.assert_array_equal(c, st.charge)
    np.testing.assert_array_equal(l, st.Lambda)
    np.testing.assert_allclose(g, st.Gamma)


def test_post_selected_bond0():
    g, l, c = engine.product_state(6, engine.lossy_single_photon_rhos(6, [0, 2, 4], 0.5, 4), 4, 16,
                                   total_photons=2)
    assert (c[0, 0] == [2, 2]).all() and (c[0, 1:] == 4).all()


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
