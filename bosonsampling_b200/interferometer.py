"""Seeded Haar-random interferometer and its Clements rectangular mesh.

The reference draws its mesh from a custom reflectivity pdf plus per-BS phase seeds
(``src/interferometer.py:9-53``); the workloads here instead use a Haar-random
unitary decomposed into a Clements rectangular mesh.  This module is written from
the published algorithm (W. R. Clements et al., "Optimal design for universal
multiport interferometers", Optica 3, 1460 (2016)):

    T_{m,m+1}(theta, phi) = [[e^{i phi} cos(theta), -sin(theta)],
                             [e^{i phi} sin(theta),  cos(theta)]]

Elements of U are nulled alternately by T^{-1} from the right (odd diagonals) and by
T from the left (even diagonals); the left factors are then commuted through the
remaining diagonal, T^{-1}(theta, phi) D = D' T(theta, phi'), so that
``U = D_out * T_K ... T_2 T_1``.  ``theta`` lies in [0, pi/2] and ``phi`` in [0, 2 pi).

The mesh is returned in application order grouped into brick-wall layers: layer
``l`` acts on pairs (m, m+1) with m of one parity, the same walk as the reference's
``LayerUpdate`` (``src/beam_splitter_parallel/Full.py:149-166``).
"""
import numpy as np


def haar_unitary(n, seed):
    """Haar unitary: complex Gaussian Z, QR, Q * diag(R_ii / |R_ii|)."""
    rng = np.random.default_rng(seed)
    z = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    ph = np.diag(r) / np.abs(np.diag(r))
    return q * ph[None, :]


def t_block(theta, phi):
    """2x2 block of T_{m,m+1}(theta, phi)."""
    c, s = np.cos(theta), np.sin(theta)
    e = np.exp(1j * phi)
    return np.array([[e * c, -s], [e * s, c]], dtype=np.complex128)


def _embed(n, m, blk):
    t = np.eye(n, dtype=np.complex128)
    t[m:m + 2, m:m + 2] = blk
    return t


def clements_decompose(U):
    """Decompose ``U`` into ``(bs_list, out_phases)``.

    ``bs_list`` is a list of ``(layer, mode, theta, phi)`` in application order and
    ``U == diag(exp(1j*out_phases)) @ T_K @ ... @ T_1``.
    """
    U = np.array(U, dtype=np.complex128)
    n = U.shape[0]
    right = []   # T applied from the right as T^{-1}: U <- U T^{-1}
    left = []    # T applied from the left:           U <- T U
    for i in range(1, n):
        if i % 2 == 1:
            for j in range(i):
                r, cm, cn = n - 1 - j, i - 1 - j, i - j
                # null U[r, cm] with columns (cm, cn):
                #   e^{-i phi} cos(theta) U[r,cm] - sin(theta) U[r,cn] = 0
                a, b = U[r, cm], U[r, cn]
                theta = np.arctan2(abs(a), abs(b))
                phi = (np.angle(a) - np.angle(b)) if abs(a) > 0 else 0.0
                tinv = np.conj(_embed(n, cm, t_block(theta, phi))).T
                U = U @ tinv
                U[r, cm] = 0.0
                right.append((cm, theta, phi))
        else:
            for j in range(1, i + 1):
                rm, rn, k = n + j - i - 2, n + j - i - 1, j - 1
                # null U[rn, k] with rows (rm, rn):
                #   e^{i phi} sin(theta) U[rm,k] + cos(theta) U[rn,k] = 0
                a, b = U[rm, k], U[rn, k]
                theta = np.arctan2(abs(b), abs(a))
                phi = (np.pi + np.angle(b) - np.angle(a)) if abs(b) > 0 else 0.0
                U = _embed(n, rm, t_block(theta, phi)) @ U
                U[rn, k] = 0.0
                left.append((rm, theta, phi))
    # U is now diagonal: D = T_Lp..T_L1 U0 T_R1^{-1}..T_Rq^{-1}
    # => U0 = T_L1^{-1}..T_Lp^{-1} D T_Rq..T_R1; commute each T_L^{-1} through D.
    alpha = np.angle(np.diag(U)).copy()
    moved = []
    for (m, theta, phi) in reversed(left):
        a, b = alpha[m], alpha[m + 1]
        # T^{-1}(theta,phi) diag(e^{ia}, e^{ib}) = diag(e^{i(b-phi+pi)}, e^{ib}) T(theta, a-b+pi)
        phi_new = a - b + np.pi
        alpha[m] = b - phi + np.pi
        moved.append((m, theta, phi_new))
    # application order: T_R1 .. T_Rq, then T'_p .. T'_1 (the order they were moved)
    seq = list(right) + moved
    # brick-wall layering by dependency (as-soon-as-possible)
    last = np.full(n, -1)
    out = []
    for (m, theta, phi) in seq:
        layer = int(max(last[m], last[m + 1]) + 1)
        last[m] = last[m + 1] = layer
        out.append((layer, m, float(theta), float(np.mod(phi, 2 * np.pi))))
    out.sort(key=lambda x: (x[0], x[1]))
    return out, np.mod(alpha, 2 * np.pi)


def mesh_unitary(n, bs_list, out_phases):
    """Rebuild the N x N unitary of a mesh (check of :func:`clements_decompose`)."""
    U = np.eye(n, dtype=np.complex128)
    for (_, m, theta, phi) in bs_list:
        U = _embed(n, m, t_block(theta, phi)) @ U
    return np.diag(np.exp(1j * np.asarray(out_phases))) @ U


def circuit(n, seed):
    """Seeded Haar unitary and its mesh: ``(U, bs_list, out_phases)``."""
    U = haar_unitary(n, seed)
    bs, ph = clements_decompose(U)
    return U, bs, ph
