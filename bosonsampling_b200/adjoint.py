"""Differentiation form: gradients of a loss on the output marginals with respect to every
beam splitter's (theta, phi) and the input transmissivity eta.

The reference simulates forward only; the update it would differentiate is
``InitializationMPO.Update`` (``src/MPO.py:234-279``): per new centre charge the block
product ``C = sum Gamma_L[a, q] w(U) Gamma_R[q, b]``, ``theta = C diag(Lambda_R)``, thin SVD
``theta = V S Y^H``, keep the top chi over all sectors, ``Gamma_L' = V``, ``Lambda' = S``,
``Gamma_R' = V^H C``.  The forward here is the library's own update (``bsmpo_bs_update`` /
``bsmpo_run_mesh`` on the device, plain FP64 path by default).  The backward is a
hand-derived adjoint of that update, run on the device:

* gauge: ``Gamma_L' Gamma_R' = V V^H C`` and ``Lambda'`` do not depend on the phases of the
  kept vectors, so the loss is gauge invariant and the adjoint needs no gauge term;
* SVD: with ``U`` the exact left vectors (the forward's kept ``V = U_k R``, so
  ``Ubar_k = Vbar R^H``), ``J = U^H Ubar``,
  ``theta_bar = U [(F o (J - J^H)) S + diag(Sbar)] Y^H + (I - U U^H) Ubar S^-1 Y^H`` over the
  whole thin spectrum (the discarded vectors enter through F), with the Lorentzian-
  broadened ``F_ij = D / (D^2 + eps_ij)``, ``D = s_j^2 - s_i^2``,
  ``eps_ij = (1e-8 max(s_i^2, s_j^2))^2``: inside an exactly degenerate multiplet -- lossy
  single photons give many -- J - J^H vanishes in exact arithmetic, and the broadening
  keeps its rounding from being multiplied by 1 / D; being relative to the pair, it leaves
  the coupling of a small kept singular value to the zero ones (rank-deficient sectors)
  intact;
* contraction: ``Gamma_L_bar[:, q] += (Cbar o conj(w_q)) Gamma_R[q, :]^H``,
  ``Gamma_R_bar[q, :] += Gamma_L[:, q]^H (Cbar o conj(w_q))``, and the gate weights' gradient
  from the block sums of ``Cbar o conj(Gamma_L[:, q] Gamma_R[q, :])``, turned into
  dL/dtheta, dL/dphi on the device (``bsmpo_bs_angle_grad``);
* memory: the forward keeps, per update, the two sites and three bonds it reads and the
  two sites and bond it writes (4 chi^2 complex numbers), not whole states.

The loss, the output phases and the marginals are plain torch operations on the device
(autograd glue); the initial product state's dependence on eta is the derivative of
its entries (1 - eta, eta).
"""
import ctypes
import math

import numpy as np

from . import _capi, engine


def _torch():
    import torch
    return torch


class StateT:
    """A device state (Gamma [n, chi, chi], Lambda [n-1, chi]) with host charges."""

    def __init__(self, G, Lam, charge, d):
        self.G, self.Lam, self.d = G, Lam, d
        self.charge = charge if isinstance(charge, np.ndarray) else charge.cpu().numpy()
        self.n, self.chi = int(G.shape[0]), int(G.shape[1])
        self._lam_host = None

    def lam_host(self, b):
        if b == 0 or b == self.n:
            return np.ones(self.chi)
        if self._lam_host is None:
            self._lam_host = self.Lam.cpu().numpy()
        return self._lam_host[b - 1]

    def lam_dev(self, b):
        torch = _torch()
        if b == 0 or b == self.n:
            return torch.ones(self.chi, dtype=torch.float64, device=self.G.device)
        return self.Lam[b - 1]

    def valid(self, b):
        return (self.charge[b, :, 0] < self.d) & (self.lam_host(b) > 0)


def state_of(sim):
    g, lam, c = sim.store()
    return StateT(g, lam, c, sim.d)


_GRIDS = {}


def _block_grid(d):
    """Charge grids (a0, a1, q0, q1, b0, b1), each of shape (d,)*6."""
    if d not in _GRIDS:
        _GRIDS[d] = np.meshgrid(*([np.arange(d)] * 6), indexing="ij")
    return _GRIDS[d]


def _block_weights(U3h, d, cc0, cc1):
    """Gate weight w[a, q, b] (a, q, b = charge blocks c0 * d + c1) of sector (cc0, cc1):
    U3[a0-cc0, cc0-b0, a0-q0] conj(U3[a1-cc1, cc1-b1, a1-q1]) where b <= q <= a and the
    rows / columns belong to the sector, else 0; with the flat U3 indices of both factors."""
    A0, A1, Q0, Q1, B0, B1 = _block_grid(d)
    ok = ((A0 >= cc0) & (A1 >= cc1) & (B0 <= cc0) & (B1 <= cc1) &
          (B0 <= Q0) & (Q0 <= A0) & (B1 <= Q1) & (Q1 <= A1))
    i0 = np.where(ok, ((A0 - cc0) * d + (cc0 - B0)) * d + (A0 - Q0), 0)
    i1 = np.where(ok, ((A1 - cc1) * d + (cc1 - B1)) * d + (A1 - Q1), 0)
    u = U3h.reshape(-1)
    w = np.where(ok, u[i0] * np.conj(u[i1]), 0.0)
    sh = (d * d, d * d, d * d)
    # axes (a0, a1, q0, q1, b0, b1) -> [a, q, b]
    return w.reshape(sh), ok.reshape(sh), i0.reshape(sh), i1.reshape(sh)


def sector_range(st, m):
    """Range of new centre charges of the update at mode m (as the forward's)."""
    d = st.d
    CL, CR = st.charge[m], st.charge[m + 2]
    vl, vr = st.valid(m), st.valid(m + 2)
    hi0 = int(CL[vl, 0].max()) if vl.any() else 0
    hi1 = int(CL[vl, 1].max()) if vl.any() else 0
    lo0 = int(CR[vr, 0].min()) if vr.any() else 0
    lo1 = int(CR[vr, 1].min()) if vr.any() else 0
    return lo0, hi0, lo1, hi1


def svd_backward(theta, V, Vbar, Sbar, eps_rel=1e-8):
    """Adjoint of the truncated thin SVD: gradient of theta (m x n) given the gradients of
    the kept left vectors (Vbar, m x k; V = the forward's kept vectors) and of the kept
    singular values (Sbar, k).  Uses the whole thin spectrum of theta, so the discarded
    singular values enter the kept vectors' terms."""
    torch = _torch()
    m, k = V.shape
    if theta.is_cuda:
        U, S, Yh = torch.linalg.svd(theta, full_matrices=False, driver="gesvdj")
    else:
        U, S, Yh = torch.linalg.svd(theta, full_matrices=False)
    r = S.shape[0]
    Y = Yh.conj().transpose(0, 1).contiguous()
    U = U.contiguous()
    Ub = torch.zeros((m, r), dtype=theta.dtype, device=theta.device)
    if k:
        # the forward's kept vectors in the SVD's basis, V = U_k R: its phases, its basis
        # inside degenerate multiplets, and the mixing of neighbouring small singular
        # vectors that an iterative forward leaves at the rounding level; the gradient
        # with respect to U_k is then Vbar R^H, and the formula below runs on the exact,
        # orthonormal singular vectors
        R = U[:, :k].conj().transpose(0, 1) @ V
        Ub[:, :k] = Vbar @ R.conj().transpose(0, 1)
    J = U.conj().transpose(0, 1) @ Ub
    s2 = S * S
    D = s2[None, :] - s2[:, None]                   # s_j^2 - s_i^2
    # broadening relative to the pair's own scale: it damps near-degenerate pairs only,
    # not the coupling of a small kept singular value to the (near-)zero ones
    eps = (eps_rel * torch.maximum(s2[None, :], s2[:, None])) ** 2
    den = D * D + eps
    F = torch.where(den > 0, D / torch.where(den > 0, den, torch.ones_like(den)), torch.zeros_like(D))
    F.fill_diagonal_(0.0)
    core = (F * (J - J.conj().transpose(0, 1))) * S[None, :].to(theta.dtype)
    core = core + torch.diag(torch.cat([Sbar, Sbar.new_zeros(r - k)]).to(theta.dtype))
    g = U @ core @ Y.conj().transpose(0, 1)
    if m > r and k:
        Ubk = Ub[:, :k]
        P = Ubk - U @ (U.conj().transpose(0, 1) @ Ubk)
        g = g + (P / S[:k][None, :].to(theta.dtype)) @ Y[:, :k].conj().transpose(0, 1)
    return g


def _qblocks(st, m):
    """Centre charge blocks (q0, q1, device index tensor) of the update at mode m."""
    torch = _torch()
    d, CC, vC = st.d, st.charge[m + 1], st.valid(m + 1)
    out = []
    for q0 in range(d):
        for q1 in range(d):
            idx = np.nonzero(vC & (CC[:, 0] == q0) & (CC[:, 1] == q1))[0]
            if len(idx):
                out.append((q0, q1, torch.as_tensor(idx, device=st.G.device)))
    return out


def update_backward(before, after, m, U3, Gbar, Lbar):
    """Backward of one update at mode m from ``before`` to ``after`` (StateT) with gate
    tensor U3 (device complex128 [d, d, d]).  Gbar [n, chi, chi] and Lbar [n-1, chi]
    (device) hold the gradients with respect to the state after the update; on return
    they hold those with respect to the state before it.  Returns the gradient of the
    gate tensor (device complex128 [d, d, d]).

    Dense per centre block q: Gamma_L with the columns outside q zeroed (GLq), Gamma_R
    with the rows outside q zeroed (GRq), X_q = GLq GRq; a sector's weights w_q expanded to
    chi x chi from the rows' and columns' charge blocks (zero outside the sector)."""
    torch = _torch()
    d, chi, n = before.d, before.chi, before.n
    dev, ct = before.G.device, before.G.dtype
    nb = d * d
    GL, GR = before.G[m], before.G[m + 1]
    lamR = before.lam_dev(m + 2)
    CL, CR = before.charge[m], before.charge[m + 2]
    vL, vR = before.valid(m), before.valid(m + 2)
    qb = _qblocks(before, m)
    if not qb:
        return torch.zeros((d, d, d), dtype=ct, device=dev)
    qids = [q0 * d + q1 for (q0, q1, _) in qb]
    cmask = torch.zeros((len(qb), chi), dtype=ct, device=dev)
    for t, (_, _, cidx) in enumerate(qb):
        cmask[t, cidx] = 1.0
    GLq = GL[None, :, :] * cmask[:, None, :]
    GRq = GR[None, :, :] * cmask[:, :, None]
    X = GLq @ GRq                                   # [Q, chi, chi]
    GLqH = GLq.conj().transpose(1, 2)
    GRqH = GRq.conj().transpose(1, 2)
    blkL = np.where(vL, CL[:, 0] * d + CL[:, 1], nb).astype(np.int64)
    blkR = np.where(vR, CR[:, 0] * d + CR[:, 1], nb).astype(np.int64)
    # outputs of the forward and the incoming gradients
    GLp = after.G[m]
    CCp, vCp = after.charge[m + 1], after.valid(m + 1)
    GbL, GbR = Gbar[m].clone(), Gbar[m + 1].clone()
    Sb_all = Lbar[m].clone() if 0 < m + 1 < n else None
    gGL = torch.zeros((chi, chi), dtype=ct, device=dev)
    gGR = torch.zeros((chi, chi), dtype=ct, device=dev)
    gLR = torch.zeros(chi, dtype=torch.float64, device=dev)
    U3h = U3.cpu().numpy()
    u_flat = U3h.reshape(-1)
    ubar = np.zeros(d ** 3, dtype=np.complex128)
    wbar_dev, wbar_meta = [], []      # block sums of the weights' gradient, read once at the end
    lo0, hi0, lo1, hi1 = sector_range(before, m)
    for cc0 in range(lo0, hi0 + 1):
        for cc1 in range(lo1, hi1 + 1):
            inL = vL & (CL[:, 0] >= cc0) & (CL[:, 1] >= cc1)
            inR = vR & (CR[:, 0] <= cc0) & (CR[:, 1] <= cc1)
            l_idx, r_idx = np.nonzero(inL)[0], np.nonzero(inR)[0]
            if not len(l_idx) or not len(r_idx):
                continue
            slots = np.nonzero(vCp & (CCp[:, 0] == cc0) & (CCp[:, 1] == cc1))[0]
            if not len(slots):
                continue                    # truncated away: no path to the loss
            li = torch.as_tensor(l_idx, device=dev)
            ri = torch.as_tensor(r_idx, device=dev)
            sl = torch.as_tensor(slots, device=dev)
            wb, ok, i0, i1 = _block_weights(U3h, d, cc0, cc1)
            wbx = np.zeros((nb + 1, len(qids), nb + 1), dtype=np.complex128)
            wbx[:nb, :, :nb] = wb[:, qids, :]
            wbx_d = torch.as_tensor(wbx, device=dev)
            rb = torch.as_tensor(np.where(inL, blkL, nb), device=dev)
            cb = torch.as_tensor(np.where(inR, blkR, nb), device=dev)
            Om = wbx_d[rb][:, :, cb].permute(1, 0, 2)   # [Q, chi, chi]
            # forward recompute of the sector
            C = (X * Om).sum(0)[li][:, ri]
            theta = C * lamR[ri][None, :]
            # gradients of the outputs: Gamma_L' = V, Gamma_R' = V^H C, Lambda' = S
            V = GLp[li][:, sl]
            Wb = GbR[sl][:, ri]
            Vb = GbL[li][:, sl] + C @ Wb.conj().transpose(0, 1)
            Sb = Sb_all[sl] if Sb_all is not None else torch.zeros(len(slots), dtype=torch.float64, device=dev)
            tb = svd_backward(theta, V, Vb, Sb)
            Cb = V @ Wb + tb * lamR[ri][None, :]
            gLR.index_add_(0, ri, (tb.conj() * C).real.sum(0))
            # contraction adjoint
            Cbf = torch.zeros((chi, chi), dtype=ct, device=dev)
            Cbf[li[:, None], ri[None, :]] = Cb
            Cw = Cbf[None] * Om.conj()
            gGL += (Cw @ GRqH).sum(0)
            gGR += (GLqH @ Cw).sum(0)
            Ra = torch.nn.functional.one_hot(rb, nb + 1).to(ct)
            Rc = torch.nn.functional.one_hot(cb, nb + 1).to(ct)
            wbar_dev.append((Ra.transpose(0, 1)[None] @ (Cbf[None] * X.conj()) @ Rc[None])[:, :nb, :nb])
            wbar_meta.append((ok[:, qids, :], i0[:, qids, :], i1[:, qids, :]))
    for wq, (okq, i0q, i1q) in zip([w.cpu().numpy() for w in wbar_dev], wbar_meta):
        # wq, okq, i0q, i1q: [a, Q, b] after the transpose below
        wq = wq.transpose(1, 0, 2)
        u0, u1 = u_flat[i0q], u_flat[i1q]
        np.add.at(ubar, i0q[okq], (wq * u1)[okq])
        np.add.at(ubar, i1q[okq], (np.conj(wq) * u0)[okq])
    Gbar[m] = gGL
    Gbar[m + 1] = gGR
    if 0 < m + 1 < n:
        Lbar[m].zero_()                     # the old centre Lambda only masks
    if m + 2 < n:
        Lbar[m + 1] += gLR
    return torch.as_tensor(ubar.reshape(d, d, d), device=dev)


# ----------------------------------------------------------------------------- observables
def _diag_masks(charge, lam_host_fn, n, d):
    return [(charge[b, :, 0] == charge[b, :, 1]) & (charge[b, :, 0] < d) & (lam_host_fn(b) > 0)
            for b in range(n + 1)]


def marginals_torch(G, charge, lam_host_fn, d):
    """(trace, P[n, d]) of the MPO Gamma_0 ... Gamma_{n-1} as differentiable torch
    operations (the same environments as the library's observables)."""
    torch = _torch()
    n = G.shape[0]
    dev, ct = G.device, G.dtype
    masks = [torch.as_tensor(mk, device=dev).to(ct) for mk in _diag_masks(charge, lam_host_fn, n, d)]
    R = [None] * (n + 1)
    R[n] = masks[n]
    for b in range(n - 1, -1, -1):
        R[b] = masks[b] * (G[b] @ R[b + 1])
    L = [None] * (n + 1)
    L[0] = masks[0]
    for b in range(n):
        L[b + 1] = masks[b + 1] * (L[b] @ G[b])
    P = []
    for i in range(n):
        occ = (charge[i, :, 0].astype(np.int64)[:, None] - charge[i + 1, :, 0].astype(np.int64)[None, :])
        M = L[i][:, None] * G[i] * R[i + 1][None, :]
        row = []
        for k in range(d):
            sel = torch.as_tensor(occ == k, device=dev)
            row.append((M * sel).sum())
        P.append(torch.stack(row))
    return R[0].sum(), torch.stack(P)


def phase_factors(charge, phases, d, device):
    """Factors e^{i phi_m (dk - db)} of the output phase screen, per site [n, chi, chi]."""
    torch = _torch()
    n = charge.shape[0] - 1
    a = charge[:-1].astype(np.int64)
    b = charge[1:].astype(np.int64)
    dk = a[:, :, None, 0] - b[:, None, :, 0]
    db = a[:, :, None, 1] - b[:, None, :, 1]
    valid = (a[:, :, None, 0] < d) & (b[:, None, :, 0] < d)
    ph = np.asarray(phases, dtype=np.float64)[:, None, None]
    f = np.where(valid, np.exp(1j * ph * (dk - db)), 1.0)
    return torch.as_tensor(f, device=device)


def marginal_loss(P, tr, target):
    """Squared L2 distance between the normalised marginals and ``target`` [n, d]."""
    return ((P.real / tr.real - target) ** 2).sum()


# ----------------------------------------------------------------------------- gates
def gate_tensor(d, theta, phi, device):
    """The mesh beam splitter's tensor U[new_a][new_b][old_a] of T(theta, phi) (as
    bsmpo_run_mesh builds it), complex128 [d, d, d] on the device."""
    torch = _torch()
    L = _capi.lib()
    c, s = math.cos(theta), math.sin(theta)
    e = complex(math.cos(phi), math.sin(phi))
    # M = T^T, T = [[e c, -s], [e s, c]]; 8 doubles (re, im of M00, M01, M10, M11)
    M = np.array([(e * c).real, (e * c).imag, (e * s).real, (e * s).imag, -s, 0.0, c, 0.0])
    u = torch.empty((d, d, d), dtype=torch.complex128, device=device)
    _capi.check(L.bsmpo_unitary(d, _capi.dptr(M), ctypes.c_void_p(u.data_ptr()),
                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), None)
    return u


def identity_tensor(d, device):
    """The tensor of the identity gate (the canonicalising sweep's)."""
    return gate_tensor(d, 0.0, 0.0, device)


def angle_grads(d, thetas, phis, ubar):
    """(dL/dtheta, dL/dphi) of every gate from its tensor gradients ubar [n_gates, d, d, d]."""
    torch = _torch()
    L = _capi.lib()
    ng = len(thetas)
    th = np.ascontiguousarray(thetas, dtype=np.float64)
    ph = np.ascontiguousarray(phis, dtype=np.float64)
    ub = ubar.to(torch.complex128).contiguous()
    out = torch.zeros((ng, 2), dtype=torch.float64, device=ub.device)
    _capi.check(L.bsmpo_bs_angle_grad(d, ng, _capi.dptr(th), _capi.dptr(ph), ctypes.c_void_p(ub.data_ptr()),
                                      ctypes.c_void_p(out.data_ptr()),
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), None)
    return out[:, 0], out[:, 1]


# ----------------------------------------------------------------------------- circuits
def _t_matrix(theta, phi):
    c, s = math.cos(theta), math.sin(theta)
    e = complex(math.cos(phi), math.sin(phi))
    return np.array([[e * c, -s], [e * s, c]], dtype=np.complex128)


class _Sites:
    """Two site tensors of a state, indexable by their site numbers."""

    def __init__(self, tensors):
        self._t = tensors
        first = next(iter(tensors.values()))
        self.device, self.dtype = first.device, first.dtype

    def __getitem__(self, i):
        return self._t[i]


class _Piece:
    """The part of a state that the update at mode m reads and writes: sites m, m+1 and
    the bonds m, m+1, m+2 (the StateT interface of update_backward)."""

    def __init__(self, st, m):
        self.d, self.chi, self.n, self.m = st.d, st.chi, st.n, m
        self.G = _Sites({m: st.G[m].clone(), m + 1: st.G[m + 1].clone()})
        self.charge = {b: st.charge[b].copy() for b in (m, m + 1, m + 2)}
        self._lam = {b: st.lam_dev(b).clone() for b in (m, m + 1, m + 2)}
        self._lam_h = {b: st.lam_host(b).copy() for b in (m, m + 1, m + 2)}

    def lam_dev(self, b):
        return self._lam[b]

    def lam_host(self, b):
        return self._lam_h[b]

    def valid(self, b):
        return (self.charge[b][:, 0] < self.d) & (self._lam_h[b] > 0)


class DiffCircuit:
    """A lossy-single-photon circuit whose output marginals are differentiable in every
    beam splitter's (theta, phi) and in eta.

    ``mesh``: (layer, mode, theta, phi) in circuit order (``interferometer.circuit``);
    ``phases``: the output phase screen (it leaves the marginals unchanged but is part of
    the forward).  The forward runs on the library (``precision``, default the plain FP64
    path), one update after another, keeping for each update the two sites and three
    bonds it reads and the two sites and bond it writes (4 chi^2 complex numbers): the
    backward needs the forward's own output basis -- inside degenerate multiplets of
    singular values the library's result is not bitwise the same between its concurrent
    and sequential schedules, so recomputing a segment from a stored MPO could hand the
    adjoint a different (equally valid) basis than the one its incoming gradient refers to."""

    def __init__(self, n, d, chi, photon_modes, mesh, phases, precision="fp64", workers=8):
        self.n, self.d, self.chi = n, d, chi
        self.photon_modes = list(photon_modes)
        self.mesh = [(int(l), int(m)) for (l, m, _, _) in mesh]
        self.phases = np.asarray(phases, dtype=np.float64)
        self.sim = engine.MPOSimulator(n, d, chi)
        self.sim.set_precision(precision)
        self.sim.set_workers(workers)
        nl = max([l for (l, _) in self.mesh] + [-1]) + 1
        self.layers = [[i for i, (l, _) in enumerate(self.mesh) if l == L] for L in range(nl)]

    def close(self):
        self.sim.close()

    # the forward, on the library only (no records)
    def run(self, thetas, phis, eta):
        """(trace, P) of the circuit with these angles, from the library's observables."""
        sim = self.sim
        sim.init_single_photons(self.photon_modes, eta)
        for L in self.layers:
            if L:
                sim.run_mesh([self.mesh[i][1] for i in L], [thetas[i] for i in L], [phis[i] for i in L])
        sim.apply_phases(self.phases)
        return sim.observables()

    def _state(self):
        g, lam, c = self.sim.store()
        return StateT(g, lam, c, self.d)

    def forward_records(self, thetas, phis, eta):
        """Runs the circuit update by update; returns the product state, the records
        (mode, gate angles or None, before, after) of every update -- the canonicalising
        sweep's and the mesh's -- and the final state."""
        sim = self.sim
        sim.init_single_photons(self.photon_modes, eta, canonicalize=False)
        prod = self._state()
        cur = prod
        recs = []
        steps = [(m, None) for m in range(self.n - 2, -1, -1)]
        steps += [(self.mesh[i][1], i) for L in self.layers for i in L]
        for (m, i) in steps:
            S = np.eye(2, dtype=np.complex128) if i is None else _t_matrix(thetas[i], phis[i])
            before = _Piece(cur, m)
            sim.bs_update(m, S)
            cur = self._state()
            recs.append((m, i, before, _Piece(cur, m)))
        return prod, recs, cur

    def backward(self, thetas, phis, eta, prod, recs, final, Gbar):
        """Gradients (theta [n_bs], phi [n_bs], eta) from Gbar = dL/dGamma of the final
        state (before the phase screen)."""
        torch = _torch()
        d, n, chi = self.d, self.n, self.chi
        dev = final.G.device
        Gbar = Gbar.clone()
        Lbar = torch.zeros((n - 1, chi), dtype=torch.float64, device=dev)
        ubar = torch.zeros((len(self.mesh), d, d, d), dtype=torch.complex128, device=dev)
        ident = identity_tensor(d, dev)
        for (m, i, before, after) in reversed(recs):
            u = ident if i is None else gate_tensor(d, thetas[i], phis[i], dev)
            ub = update_backward(before, after, m, u, Gbar, Lbar)
            if i is not None:
                ubar[i] = ub
        # eta: the product state's entries are (1 - eta) at occupation (0, 0) and eta at
        # (1, 1) on the photon modes
        g_eta = 0.0
        for i in self.photon_modes:
            a = prod.charge[i].astype(np.int64)
            b = prod.charge[i + 1].astype(np.int64)
            ok = (a[:, None, 0] < d) & (b[None, :, 0] < d)
            o0 = a[:, None, 0] - b[None, :, 0]
            o1 = a[:, None, 1] - b[None, :, 1]
            dG = np.where(ok & (o0 == 0) & (o1 == 0), -1.0, 0.0) + np.where(ok & (o0 == 1) & (o1 == 1), 1.0, 0.0)
            g_eta += float((Gbar[i].real * torch.as_tensor(dG, device=dev)).sum())
        g_th, g_ph = angle_grads(d, thetas, phis, ubar)
        return g_th, g_ph, g_eta

    def loss_and_grad(self, thetas, phis, eta, target):
        """(loss, dL/dtheta, dL/dphi, dL/deta) of the marginal loss against ``target``."""
        torch = _torch()
        prod, recs, final = self.forward_records(thetas, phis, eta)
        G = final.G.clone().requires_grad_(True)
        f = phase_factors(final.charge, self.phases, self.d, G.device)
        tr, P = marginals_torch(G * f, final.charge, final.lam_host, self.d)
        tgt = torch.as_tensor(np.asarray(target, dtype=np.float64), device=G.device)
        loss = marginal_loss(P, tr, tgt)
        loss.backward()
        g_th, g_ph, g_eta = self.backward(thetas, phis, eta, prod, recs, final, G.grad)
        return float(loss.detach()), g_th, g_ph, g_eta


class CircuitMarginals:
    """``torch.autograd.Function`` form: ``CircuitMarginals.apply(thetas, phis, eta,
    circuit)`` returns (trace, P [n, d]) of a :class:`DiffCircuit`; any loss built on them
    backpropagates through the adjoint into the three parameter tensors."""

    @staticmethod
    def apply(thetas, phis, eta, circuit):
        return _marginals_function().apply(thetas, phis, eta, circuit)


_FN = None


def _marginals_function():
    global _FN
    if _FN is None:
        torch = _torch()

        class _Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, thetas, phis, eta, circuit):
                th = thetas.detach().cpu().numpy().astype(np.float64)
                ph = phis.detach().cpu().numpy().astype(np.float64)
                e = float(eta.detach())
                prod, recs, final = circuit.forward_records(th, ph, e)
                ctx.saved = (circuit, th, ph, e, prod, recs, final)
                f = phase_factors(final.charge, circuit.phases, circuit.d, final.G.device)
                with torch.no_grad():
                    tr, P = marginals_torch(final.G * f, final.charge, final.lam_host, circuit.d)
                return tr, P

            @staticmethod
            def backward(ctx, g_tr, g_P):
                circuit, th, ph, e, prod, recs, final = ctx.saved
                with torch.enable_grad():
                    G = final.G.clone().requires_grad_(True)
                    f = phase_factors(final.charge, circuit.phases, circuit.d, G.device)
                    tr, P = marginals_torch(G * f, final.charge, final.lam_host, circuit.d)
                    torch.autograd.backward([tr, P], [g_tr, g_P])
                g_th, g_ph, g_eta = circuit.backward(th, ph, e, prod, recs, final, G.grad)
                dev = g_P.device
                return (g_th.to(dev), g_ph.to(dev), torch.tensor(g_eta, dtype=torch.float64, device=dev), None)

        _FN = _Fn
    return _FN
