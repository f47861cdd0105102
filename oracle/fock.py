"""Two-mode Fock-space beam-splitter tensor (CPU oracle, test infrastructure only).

Restates the amplitude formula of the reference's ``Rand_BS_MPS`` (``src/MPO.py:6-18``)
and ``unitary`` kernel (``src/u_kernel.cu:37-71``), generalised from the reference's
(t, r) parametrisation to an arbitrary 2x2 single-particle matrix ``M``.

Convention (the reference's): ``M`` maps creation operators column-wise,
``a^+ -> M[0,0] a^+ + M[1,0] b^+`` and ``b^+ -> M[0,1] a^+ + M[1,1] b^+``; the
reference's (t, r) corresponds to ``M = [[t, -conj(r)], [r, conj(t)]]``.  The tensor

    U[n, m, l] = <l, n+m-l| Gamma(M) |n, m>
               = sqrt(l! (n+m-l)! / (n! m!)) *
                 sum_k C(n,k) C(m,l-k) M00^k M10^(n-k) M01^(l-k) M11^(m-l+k)

is stored for 0 <= n, m, l < d with 0 <= n+m-l < d (zero elsewhere).  The update
(``src/MPO.py:254``, ``src/update_MPO_kernel.cu:451``) indexes it as
``U[new_a, new_b, old_a]``, i.e. it applies Gamma(M)^T = Gamma(M^T) to the ket.
So to apply a single-particle unitary ``S`` to the state one passes ``M = S^T``
(:func:`update_tensor`).
"""
from math import comb, factorial, sqrt

import numpy as np


def bs_tensor(M, d):
    """U[n, m, l] for the single-particle matrix ``M`` (reference formula, complex128)."""
    M = np.asarray(M, dtype=np.complex128)
    m00, m01, m10, m11 = M[0, 0], M[0, 1], M[1, 0], M[1, 1]
    U = np.zeros((d, d, d), dtype=np.complex128)
    for n in range(d):
        for m in range(d):
            # photon number on the first output mode (src/MPO.py:15)
            for l in range(max(0, n + m + 1 - d), min(d, n + m + 1)):
                norm = sqrt(factorial(l) * factorial(n + m - l) / (factorial(n) * factorial(m)))
                acc = 0j
                for k in range(max(0, l - m), min(l, n) + 1):
                    acc += (comb(n, k) * comb(m, l - k) * m00 ** k * m10 ** (n - k)
                            * m01 ** (l - k) * m11 ** (m - l + k))
                U[n, m, l] = norm * acc
    return U


def tr_matrix(t, r):
    """Single-particle matrix of the reference's (t, r) beam splitter (``src/MPO.py:11``)."""
    return np.array([[t, -np.conj(r)], [r, np.conj(t)]], dtype=np.complex128)


def update_tensor(S, d):
    """Tensor the update consumes to apply the single-particle unitary ``S`` to the state.

    ``S`` acts on the one-photon amplitudes of (mode, mode+1): a photon entering mode j
    leaves mode i with amplitude ``S[i, j]``.  Returns ``bs_tensor(S.T, d)``.
    """
    return bs_tensor(np.asarray(S, dtype=np.complex128).T, d)


def reference_random_tensor(seed, d, reflectivity):
    """Restates ``Rand_BS_MPS(seed, d, r)`` (``src/MPO.py:6-18``) in complex128.

    Draws the two phases from ``np.random.RandomState(seed)`` exactly as the reference
    does and returns the 3-index tensor ``U[n, m, l]`` (the reference's 4th index is
    ``n+m-l``).
    """
    rs = np.random.RandomState(seed)
    t = np.sqrt(1 - reflectivity ** 2) * np.exp(1j * rs.rand() * 2 * np.pi)
    r = reflectivity * np.exp(1j * rs.rand() * 2 * np.pi)
    return bs_tensor(tr_matrix(t, r), d)


def tensor3_to_4(U3):
    """Expand U[n, m, l] to the reference's 4-index layout U4[n, m, l, n+m-l]."""
    d = U3.shape[0]
    U4 = np.zeros((d,) * 4, dtype=U3.dtype)
    for n in range(d):
        for m in range(d):
            for l in range(d):
                o = n + m - l
                if 0 <= o < d:
                    U4[n, m, l, o] = U3[n, m, l]
    return U4


def tensor4_to_3(U4):
    """Inverse of :func:`tensor3_to_4`."""
    d = U4.shape[0]
    U3 = np.zeros((d, d, d), dtype=U4.dtype)
    for n in range(d):
        for m in range(d):
            for l in range(d):
                o = n + m - l
                if 0 <= o < d:
                    U3[n, m, l] = U4[n, m, l, o]
    return U3
