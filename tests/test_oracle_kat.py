"""Known answers for the CPU oracle (no reference run needed)."""
import numpy as np
import pytest
from scipy.stats import binom

from oracle import circuit, fock, interferometer as itf, mpo


@pytest.mark.parametrize("d", [3, 4, 5])
def test_bs_tensor_unitary_per_photon_block(d):
    U3 = fock.update_tensor(itf.t_block(0.7, 1.3), d)
    for N in range(d):
        idx = [(n, N - n) for n in range(N + 1)]
        M = np.array([[U3[a[0], a[1], b[0]] for b in idx] for a in idx])
        np.testing.assert_allclose(M @ M.conj().T, np.eye(N + 1), atol=1e-14)


def test_tensor_layout_roundtrip():
    U3 = fock.reference_random_tensor(7, 4, 0.5)
    np.testing.assert_array_equal(fock.tensor4_to_3(fock.tensor3_to_4(U3)), U3)


@pytest.mark.parametrize("n,eta,d", [(16, 0.5, 4), (8, 0.5, 4), (10, 0.3, 5)])
def test_trace_is_binomial_cdf(n, eta, d):
    st = mpo.initial_state(n, circuit.even_modes(n), eta, d, 64)
    assert abs(mpo.trace(st) - binom.cdf(d - 1, len(circuit.even_modes(n)), eta)) < 1e-13


def test_single_photon_marginals_follow_the_unitary():
    n = 6
    U, bs, ph = itf.circuit(n, 7)
    for j in (0, 3):
        st = mpo.initial_state(n, [j], 0.8, 2, 16)
        for (l, m, th, p) in bs:
            mpo.bs_update(st, m, fock.update_tensor(itf.t_block(th, p), 2))
        P = mpo.marginals(st)
        np.testing.assert_allclose(P[:, 1].real, 0.8 * np.abs(U[:, j]) ** 2, atol=1e-13)


def test_hong_ou_mandel_dip():
    st = mpo.initial_state(2, [0, 1], 1.0, 3, 9)
    mpo.bs_update(st, 0, fock.update_tensor(itf.t_block(np.pi / 4, 0.0), 3))
    P = mpo.marginals(st)
    assert abs(P[0, 1]) < 1e-15
    np.testing.assert_allclose(P[0].real, [0.5, 0, 0.5], atol=1e-14)


def test_trace_conserved_without_truncation():
    n, d = 8, 3
    U, bs, ph = itf.circuit(n, 3)
    st = mpo.initial_state(n, range(0, n, 2), 0.5, d, 81)
    t0 = mpo.trace(st)
    for (l, m, th, p) in bs:
        mpo.bs_update(st, m, fock.update_tensor(itf.t_block(th, p), d))
    assert abs(mpo.trace(st) - t0) < 1e-12
    P = mpo.marginals(st)
    np.testing.assert_allclose(P.sum(axis=1), np.full(n, t0), atol=1e-12)


def test_truncation_keeps_hermitian_pairs_together():
    st, U, bs = circuit.run(**circuit.WORKLOADS["plain-small"], max_bs=40)
    from collections import Counter
    for b in range(1, st.n):
        valid = st.charge[b, :, 0] < st.d
        cnt = Counter(map(tuple, st.charge[b][valid].tolist()))
        assert all(cnt[(x, y)] == cnt[(y, x)] for (x, y) in cnt)
    assert abs(mpo.trace(st).imag) < 1e-14
