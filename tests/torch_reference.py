"""Pure-torch FP64 autograd reference of the circuit (test infrastructure only).

The oracle's update (``oracle/mpo.py:bs_update``, restating ``src/MPO.py:158-303``)
written with torch operations, so that torch autograd differentiates the whole circuit --
product state in eta, Fock tensors in (theta, phi), contraction, thin SVD of every sector
(``torch.linalg.svd``), top-chi truncation (the oracle's selection on the detached
singular values), phase screen and marginals.  It is the checker of the library's
hand-written adjoint (``bosonsampling_b200.adjoint``); small configurations only.
"""
from math import comb, factorial, sqrt

import numpy as np
import torch

from oracle import mpo as om


def fock_tensor(M, d):
    """U[n, m, l] of the single-particle matrix M (2 x 2 complex torch tensor), the
    oracle's formula (``oracle/fock.py:bs_tensor``), differentiable in M."""
    m00, m01, m10, m11 = M[0, 0], M[0, 1], M[1, 0], M[1, 1]
    vals = []
    for n in range(d):
        for m in range(d):
            for l in range(d):
                o = n + m - l
                if not (0 <= o < d):
                    vals.append(torch.zeros((), dtype=torch.complex128))
                    continue
                norm = sqrt(factorial(l) * factorial(o) / (factorial(n) * factorial(m)))
                acc = torch.zeros((), dtype=torch.complex128)
                for k in range(max(0, l - m), min(l, n) + 1):
                    acc = acc + comb(n, k) * comb(m, l - k) * m00 ** k * m10 ** (n - k) * m01 ** (l - k) * m11 ** (m - l + k)
                vals.append(norm * acc)
    return torch.stack(vals).reshape(d, d, d)


def gate(theta, phi, d):
    """The mesh beam splitter's tensor: T(theta, phi) = [[e^{i phi} c, -s], [e^{i phi} s, c]], M = T^T."""
    e = torch.exp(1j * phi.to(torch.complex128))
    c, s = torch.cos(theta).to(torch.complex128), torch.sin(theta).to(torch.complex128)
    T = torch.stack([torch.stack([e * c, -s]), torch.stack([e * s, c])])
    return fock_tensor(T.transpose(0, 1), d)


class TState:
    def __init__(self, n, d, chi, G, Lam, charge):
        self.n, self.d, self.chi, self.G, self.Lam, self.charge = n, d, chi, G, Lam, charge

    def lam(self, b):
        if b == 0 or b == self.n:
            return torch.ones(self.chi, dtype=torch.float64)
        return self.Lam[b - 1]


def product_state(n, d, chi, photon_modes, eta):
    """The oracle's product state with rho = diag(1 - eta, eta) on the photon modes."""
    pm = set(photon_modes)
    ref = om.product_state(n, [om.single_photon_rho(d, 0.5) if i in pm else om.vacuum_rho(d) for i in range(n)], d, chi)
    G = []
    for i in range(n):
        a = ref.charge[i].astype(np.int64)
        b = ref.charge[i + 1].astype(np.int64)
        ok = (a[:, None, 0] < d) & (b[None, :, 0] < d)
        o0, o1 = a[:, None, 0] - b[None, :, 0], a[:, None, 1] - b[None, :, 1]
        z = torch.zeros((chi, chi), dtype=torch.complex128)
        m00 = torch.as_tensor(ok & (o0 == 0) & (o1 == 0))
        m11 = torch.as_tensor(ok & (o0 == 1) & (o1 == 1))
        if i in pm:
            g = z + m00 * (1 - eta) + m11 * eta
        else:
            g = z + m00 * 1.0
        G.append(g)
    return TState(n, d, chi, torch.stack(G), torch.as_tensor(ref.Lambda), ref.charge.copy())


def bs_update(st, mode, U3):
    """The oracle's update with torch operations (returns a new TState)."""
    d, chi, n = st.d, st.chi, st.n
    CL, CC, CR = st.charge[mode], st.charge[mode + 1], st.charge[mode + 2]
    LLh, LCh, LRh = (st.lam(b).detach().numpy() for b in (mode, mode + 1, mode + 2))
    idx_L, idx_C, idx_R = om._blocks(CL, LLh, d), om._blocks(CC, LCh, d), om._blocks(CR, LRh, d)
    GL, GR = st.G[mode], st.G[mode + 1]
    LR = st.lam(mode + 2)
    lo0, hi0, lo1, hi1 = om.sector_range(CL, CR, d, LLh, LRh)
    sectors, sig, secV, secW, secl, secr = [], [], [], [], [], []
    for cc0 in range(lo0, hi0 + 1):
        for cc1 in range(lo1, hi1 + 1):
            lblk = [(i, j) for i in range(cc0, d) for j in range(cc1, d) if len(idx_L[(i, j)])]
            rblk = [(i, j) for i in range(cc0 + 1) for j in range(cc1 + 1) if len(idx_R[(i, j)])]
            l_bond = np.concatenate([idx_L[b] for b in lblk]) if lblk else np.zeros(0, int)
            r_bond = np.concatenate([idx_R[b] for b in rblk]) if rblk else np.zeros(0, int)
            if len(l_bond) == 0 or len(r_bond) == 0:
                continue
            rows = []
            for (a0, a1) in lblk:
                la = torch.as_tensor(idx_L[(a0, a1)])
                cols = []
                for (b0, b1) in rblk:
                    rb = torch.as_tensor(idx_R[(b0, b1)])
                    blk = torch.zeros((len(la), len(rb)), dtype=torch.complex128)
                    for q0 in range(b0, a0 + 1):
                        for q1 in range(b1, a1 + 1):
                            qc = idx_C[(q0, q1)]
                            if len(qc) == 0:
                                continue
                            qc = torch.as_tensor(qc)
                            w = U3[a0 - cc0, cc0 - b0, a0 - q0] * torch.conj(U3[a1 - cc1, cc1 - b1, a1 - q1])
                            blk = blk + (GL[la][:, qc] * w) @ GR[qc][:, rb]
                    cols.append(blk)
                rows.append(torch.cat(cols, dim=1))
            C = torch.cat(rows, dim=0)
            theta = C * LR[torch.as_tensor(r_bond)][None, :]
            V, s, _ = torch.linalg.svd(theta, full_matrices=False)
            sd = s.detach().numpy()
            floor = 16.0 * np.finfo(np.float64).eps * np.sqrt(max(theta.shape)) * float(torch.linalg.norm(theta.detach()))
            s = torch.where(s <= floor, torch.zeros_like(s), s)
            sd = np.where(sd <= floor, 0.0, sd)
            W = V.conj().transpose(0, 1) @ C
            sectors.append((cc0, cc1))
            sig.append((s, sd))
            secV.append(V)
            secW.append(W)
            secl.append(l_bond)
            secr.append(r_bond)
    sig_np = [x[1] for x in sig]
    keys = om.selection_keys(sectors, sig_np)
    kept = om.select_top(sectors, keys, chi, 0.0, sig_np)
    GLo = torch.zeros((chi, chi), dtype=torch.complex128)
    GRo = torch.zeros((chi, chi), dtype=torch.complex128)
    lam = torch.zeros(chi, dtype=torch.float64)
    chg = np.full((chi, 2), d, dtype=np.int32)
    slot = 0
    for s_i, k in enumerate(kept):
        if k == 0:
            continue
        cols = torch.arange(slot, slot + k)
        li = torch.as_tensor(secl[s_i])
        ri = torch.as_tensor(secr[s_i])
        GLo = GLo.index_put((li[:, None], cols[None, :]), secV[s_i][:, :k])
        GRo = GRo.index_put((cols[:, None], ri[None, :]), secW[s_i][:k, :])
        lam = lam.index_put((cols,), sig[s_i][0][:k])
        chg[slot:slot + k] = sectors[s_i]
        slot += k
    G = torch.cat([st.G[:mode], GLo[None], GRo[None], st.G[mode + 2:]])
    Lam = torch.cat([st.Lam[:mode], lam[None], st.Lam[mode + 1:]])
    charge = st.charge.copy()
    charge[mode + 1] = chg
    return TState(n, d, chi, G, Lam, charge), kept


def canonicalize(st):
    ident = fock_tensor(torch.eye(2, dtype=torch.complex128), st.d)
    for mode in range(st.n - 2, -1, -1):
        st, _ = bs_update(st, mode, ident)
    return st


def marginals(st, phases):
    """(trace, P) after the phase screen, independent of the library's glue."""
    n, d = st.n, st.d
    G = []
    for m in range(n):
        a = st.charge[m].astype(np.int64)
        b = st.charge[m + 1].astype(np.int64)
        dk = a[:, None, 0] - b[None, :, 0]
        db = a[:, None, 1] - b[None, :, 1]
        valid = (a[:, None, 0] < d) & (b[None, :, 0] < d)
        f = torch.as_tensor(np.where(valid, np.exp(1j * phases[m] * (dk - db)), 1.0))
        G.append(st.G[m] * f)

    def mask(b):
        c = st.charge[b]
        return torch.as_tensor((c[:, 0] == c[:, 1]) & (c[:, 0] < d) & (st.lam(b).detach().numpy() > 0)).to(torch.complex128)

    R = [None] * (n + 1)
    R[n] = mask(n)
    for b in range(n - 1, -1, -1):
        R[b] = mask(b) * (G[b] @ R[b + 1])
    L = [None] * (n + 1)
    L[0] = mask(0)
    for b in range(n):
        L[b + 1] = mask(b + 1) * (L[b] @ G[b])
    P = []
    for i in range(n):
        occ = st.charge[i, :, 0].astype(np.int64)[:, None] - st.charge[i + 1, :, 0].astype(np.int64)[None, :]
        M = L[i][:, None] * G[i] * R[i + 1][None, :]
        P.append(torch.stack([M[torch.as_tensor(occ == k)].sum() for k in range(d)]))
    return R[0].sum(), torch.stack(P)


def circuit(n, d, chi, photon_modes, eta, mesh, thetas, phis, phases):
    """(trace, P) of the whole circuit as a torch graph in (thetas, phis, eta)."""
    st = canonicalize(product_state(n, d, chi, photon_modes, eta))
    for i, (_, mode, _, _) in enumerate(mesh):
        st, _ = bs_update(st, mode, gate(thetas[i], phis[i], d))
    return marginals(st, phases)
