"""Density-matrix MPO state, beam-splitter update and observables (CPU oracle).

TEST INFRASTRUCTURE ONLY -- a complex128 numpy restatement of the reference's CPU
algorithm; the product path never imports it.

State layout (the reference's after ``Initialize``, ``src/MPO.py:114-132``, embedded
into chi-sized arrays as in ``src/beam_splitter_parallel/Full.py:56-63``):

* ``Gamma[n, chi, chi]`` complex128 -- Gamma[site][left bond, right bond];
  the MPO is the plain product Gamma_0 ... Gamma_{n-1}.
* ``Lambda[n-1, chi]`` float64 -- Lambda[i] lives on bond i+1 (between sites i, i+1).
* ``charge[n+1, chi, 2]`` int32 -- (ket, bra) photons to the right of the bond,
  each <= d-1, sorted lexicographically; empty slots carry the sentinel ``d``.
  The physical occupation of site i is charge[i] - charge[i+1] (ket and bra).

Deliberate, documented differences from the reference's ``InitializationMPO.Update``:

1. sectors are indexed by loop order (``src/MPO.py:288`` uses ``i*d+j``, which is
   only right when both charge ranges are the full ``0..d-1``);
2. top-chi selection is deterministic: key = singular value (made identical within a
   ket/bra-swapped sector pair, which Hermiticity makes degenerate), ties broken by
   sector loop order then in-sector index (the reference's argpartition order is
   arbitrary), and a cut that splits such a degenerate pair keeps neither member
   (the reference keeps an arbitrary one, which breaks rho = rho^H);
3. the new bond is stored sorted by charge (the GPU driver's lexsort,
   ``src/beam_splitter_parallel/Rank.py:182-196``), empty slots get the sentinel d;
4. only singular values > 0 are candidates -- the reference keeps exact zeros but then
   masks them out everywhere through Lambda > 0 (``src/MPO.py:184-188``);
5. singular values at or below the numerical-rank floor 16 eps sqrt(max(m, n))
   ||theta||_F count as exact zeros: they are rounding noise of a rank-deficient
   sector, whose singular vectors are arbitrary (the reference, in complex64, keeps
   such noise vectors as bond entries).
"""
from dataclasses import dataclass, field

import numpy as np

from . import fock


@dataclass
class MPOState:
    n: int
    d: int
    chi: int
    Gamma: np.ndarray
    Lambda: np.ndarray
    charge: np.ndarray

    def copy(self):
        return MPOState(self.n, self.d, self.chi, self.Gamma.copy(), self.Lambda.copy(),
                        self.charge.copy())


@dataclass
class UpdateInfo:
    """Diagnostics of one BS update (per sector in loop order)."""
    sectors: list = field(default_factory=list)      # (cc0, cc1)
    sigma: list = field(default_factory=list)        # singular values, descending
    shape: list = field(default_factory=list)        # (|L_s|, |R_s|)
    kept: list = field(default_factory=list)         # kept count per sector
    trunc_weight: float = 0.0                        # sum of discarded sigma^2
    flops_gemm: float = 0.0                          # 8 * sum n_a n_q n_b over valid triples


def _edge(chi):
    return np.ones(chi, dtype=np.float64)


def bond_lambda(st, b):
    """Lambda on bond b (edges: ones)."""
    if b == 0 or b == st.n:
        return _edge(st.chi)
    return st.Lambda[b - 1]


def product_state(n_modes, rho_sites, d, chi, total_photons=None):
    """Product-state MPO with the U(1) charge structure (restates ``src/MPO.py:56-109``).

    ``rho_sites[i]`` is the d x d density matrix of input mode i.  Bond charges are the
    (ket, bra) photon numbers to the right of the bond, capped at d-1 (the reference's
    global photon cutoff).  ``total_photons`` restricts bond 0 to one charge (the
    reference's post-selected photon number, ``src/MPO.py:62-65``).
    """
    bonds = [None] * (n_modes + 1)
    bonds[n_modes] = [(0, 0)]
    for b in range(n_modes - 1, -1, -1):
        rho = rho_sites[b]
        s = set()
        for (c0, c1) in bonds[b + 1]:
            for o0 in range(d):
                for o1 in range(d):
                    if rho[o0, o1] != 0 and c0 + o0 <= d - 1 and c1 + o1 <= d - 1:
                        s.add((c0 + o0, c1 + o1))
        if b == 0:
            # bond 0 lists every diagonal total (c, c), c < d, reachable or not
            # (src/MPO.py:57-65); unreachable ones get zero rows
            if total_photons is None:
                s = {(c, c) for c in range(d)}
            else:
                s = {(total_photons, total_photons)}
        bonds[b] = sorted(s)
        if len(bonds[b]) > chi:
            raise ValueError("chi smaller than the product-state bond dimension")
    Gamma = np.zeros((n_modes, chi, chi), dtype=np.complex128)
    Lambda = np.zeros((n_modes - 1, chi), dtype=np.float64)
    charge = np.full((n_modes + 1, chi, 2), d, dtype=np.int32)
    for b in range(n_modes + 1):
        for i, c in enumerate(bonds[b]):
            charge[b, i] = c
        if 0 < b < n_modes:
            Lambda[b - 1, :len(bonds[b])] = 1.0
    for site in range(n_modes):
        rho = rho_sites[site]
        for i, (a0, a1) in enumerate(bonds[site]):
            for j, (b0, b1) in enumerate(bonds[site + 1]):
                o0, o1 = a0 - b0, a1 - b1
                if 0 <= o0 < d and 0 <= o1 < d:
                    Gamma[site, i, j] = rho[o0, o1]
    return MPOState(n_modes, d, chi, Gamma, Lambda, charge)


def single_photon_rho(d, eta):
    """(1-eta)|0><0| + eta|1><1| (the reference's 'loss' is the vacuum weight 1-eta)."""
    rho = np.zeros((d, d), dtype=np.complex128)
    rho[0, 0] = 1.0 - eta
    if d > 1:
        rho[1, 1] = eta
    return rho


def vacuum_rho(d):
    rho = np.zeros((d, d), dtype=np.complex128)
    rho[0, 0] = 1.0
    return rho


def initial_state(n_modes, photon_modes, eta, d, chi, total_photons=None):
    """Lossy single photons in ``photon_modes``, vacuum elsewhere, canonicalised.

    Generalises ``Initialize('Single photon', ...)`` (``src/MPO.py:21-134``) to arbitrary
    input modes.  The canonicalising right-to-left sweep (``src/MPO.py:137-155``) is run
    with the identity gate; the reference uses a phase-only gate (``src/MPO.py:151``),
    which acts as the identity on these diagonal input states.
    """
    pm = set(int(m) for m in photon_modes)
    rhos = [single_photon_rho(d, eta) if i in pm else vacuum_rho(d) for i in range(n_modes)]
    st = product_state(n_modes, rhos, d, chi, total_photons)
    canonicalize(st)
    return st


def canonicalize(st):
    ident = fock.bs_tensor(np.eye(2), st.d)
    for mode in range(st.n - 2, -1, -1):
        bs_update(st, mode, ident)
    return st


def _blocks(charge, lam, d):
    """Index lists per (c0, c1) charge block of one bond (``src/MPO.py:182-189``)."""
    out = {}
    for i in range(d):
        for j in range(d):
            out[(i, j)] = np.nonzero((charge[:, 0] == i) & (charge[:, 1] == j) & (lam > 0))[0]
    return out


def sector_range(CL, CR, d, lamL, lamR):
    """Range of new centre charges (``src/MPO.py:191-204``) over the valid bond entries."""
    vl = (CL[:, 0] != d) & (lamL > 0)
    vr = (CR[:, 0] != d) & (lamR > 0)
    hi0 = int(CL[vl, 0].max()) if vl.any() else 0
    hi1 = int(CL[vl, 1].max()) if vl.any() else 0
    lo0 = int(CR[vr, 0].min()) if vr.any() else 0
    lo1 = int(CR[vr, 1].min()) if vr.any() else 0
    return lo0, hi0, lo1, hi1


def selection_keys(sectors, sigmas):
    """Truncation keys: sigma, with ket/bra-swapped sector pairs made exactly equal.

    Hermiticity of rho makes sector (x, y) and (y, x) degenerate; rounding would
    otherwise decide which member of a pair survives a cut that splits it.
    """
    pos = {s: i for i, s in enumerate(sectors)}
    keys = []
    for i, (x, y) in enumerate(sectors):
        k = sigmas[i].copy()
        j = pos.get((y, x))
        if j is not None and j != i:
            p = min(len(k), len(sigmas[j]))
            k[:p] = np.maximum(k[:p], sigmas[j][:p])
        keys.append(k)
    return keys


def select_top(sectors, keys, chi, thr=0.0, sigmas=None):
    """Deterministic top-chi: returns kept count per sector (a prefix of each sector).

    Entries are ranked by key (descending), then sector loop order, then in-sector
    index.  A cut that falls inside a ket/bra-swapped pair (equal keys) keeps neither
    member, so the kept set stays closed under the swap and the MPO stays Hermitian.
    """
    entries = []
    for s, k in enumerate(keys):
        for i, v in enumerate(k):
            if v > thr and v > 0:
                entries.append((-float(v), s, i))
    entries.sort()
    kept = [0] * len(keys)
    for (_, s, i) in entries[:chi]:
        kept[s] = max(kept[s], i + 1)
    if sigmas is not None:
        # a kept vector needs its own singular value > 0 (the key may be the partner's)
        kept = [min(k, int(np.sum(sg > 0))) for k, sg in zip(kept, sigmas)]
    pos = {sec: i for i, sec in enumerate(sectors)}
    for s, (x, y) in enumerate(sectors):
        j = pos.get((y, x))
        if j is not None and j != s:
            m = min(kept[s], kept[j])
            kept[s] = kept[j] = m
    return kept


def bs_update(st, mode, U3, info=None, cutoff=0.0):
    """Apply the two-site gate with tensor ``U3[new_a, new_b, old_a]`` on (mode, mode+1).

    Restates ``InitializationMPO.Update`` (``src/MPO.py:158-303``): per new centre charge
    (cc0, cc1) the block product ``Gamma_L[a, q] diag(U (x) U*) Gamma_R[q, b]`` over valid
    charge triples a >= q >= b (``src/MPO.py:234-254``), ``theta = C diag(Lambda_R)``
    (``:256``), thin SVD (``:258``), ``W = V^H C`` (``:261``), top-chi truncation
    (``:272-279``) and scatter (``:286-303``).  ``cutoff`` > 0 additionally drops
    singular values <= cutoff * (largest singular value of the update).
    """
    d, chi, n = st.d, st.chi, st.n
    CL, CC, CR = st.charge[mode], st.charge[mode + 1], st.charge[mode + 2]
    LL, LC, LR = bond_lambda(st, mode), bond_lambda(st, mode + 1), bond_lambda(st, mode + 2)
    idx_L = _blocks(CL, LL, d)
    idx_C = _blocks(CC, LC, d)
    idx_R = _blocks(CR, LR, d)
    GL, GR = st.Gamma[mode], st.Gamma[mode + 1]
    lo0, hi0, lo1, hi1 = sector_range(CL, CR, d, LL, LR)
    if info is None:
        info = UpdateInfo()
    sec_V, sec_W, sec_l, sec_r = [], [], [], []
    for cc0 in range(lo0, hi0 + 1):
        for cc1 in range(lo1, hi1 + 1):
            lblk = [(i, j) for i in range(cc0, d) for j in range(cc1, d) if len(idx_L[(i, j)])]
            rblk = [(i, j) for i in range(cc0 + 1) for j in range(cc1 + 1) if len(idx_R[(i, j)])]
            l_bond = np.concatenate([idx_L[b] for b in lblk]) if lblk else np.zeros(0, int)
            r_bond = np.concatenate([idx_R[b] for b in rblk]) if rblk else np.zeros(0, int)
            if len(l_bond) == 0 or len(r_bond) == 0:
                continue
            C = np.zeros((len(l_bond), len(r_bond)), dtype=np.complex128)
            lo = 0
            for (a0, a1) in lblk:
                la = idx_L[(a0, a1)]
                ro = 0
                for (b0, b1) in rblk:
                    rb = idx_R[(b0, b1)]
                    cb, w = [], []
                    for q0 in range(b0, a0 + 1):
                        for q1 in range(b1, a1 + 1):
                            qc = idx_C[(q0, q1)]
                            if len(qc) == 0:
                                continue
                            wq = U3[a0 - cc0, cc0 - b0, a0 - q0] * np.conj(U3[a1 - cc1, cc1 - b1, a1 - q1])
                            cb.append(qc)
                            w.append(np.full(len(qc), wq))
                            info.flops_gemm += 8.0 * len(la) * len(qc) * len(rb)
                    if cb:
                        cb = np.concatenate(cb)
                        w = np.concatenate(w)
                        C[lo:lo + len(la), ro:ro + len(rb)] += (GL[np.ix_(la, cb)] * w[None, :]) @ GR[np.ix_(cb, rb)]
                    ro += len(rb)
                lo += len(la)
            theta = C * LR[r_bond][None, :]
            V, s, _ = np.linalg.svd(theta, full_matrices=False)
            # numerical rank: singular values <= 16 eps sqrt(max(m, n)) ||theta||_F are
            # rounding noise of a rank-deficient block and count as exact zeros
            floor = 16.0 * np.finfo(np.float64).eps * np.sqrt(max(theta.shape)) * np.linalg.norm(theta)
            s = np.where(s <= floor, 0.0, s)
            W = np.conj(V.T) @ C
            info.sectors.append((cc0, cc1))
            info.sigma.append(s)
            info.shape.append((len(l_bond), len(r_bond)))
            sec_V.append(V)
            sec_W.append(W)
            sec_l.append(l_bond)
            sec_r.append(r_bond)
    keys = selection_keys(info.sectors, info.sigma)
    smax = max([float(x[0]) for x in info.sigma if len(x)] + [0.0])
    kept = select_top(info.sectors, keys, chi, cutoff * smax, info.sigma)
    info.kept = kept
    info.trunc_weight = float(sum(float(np.sum(s[k:] ** 2)) for s, k in zip(info.sigma, kept)))
    # scatter in sector (= charge) order, each sector's kept prefix in sigma order
    GLo = np.zeros((chi, chi), dtype=np.complex128)
    GRo = np.zeros((chi, chi), dtype=np.complex128)
    lam = np.zeros(chi, dtype=np.float64)
    chg = np.full((chi, 2), d, dtype=np.int32)
    slot = 0
    for s_i, k in enumerate(kept):
        if k == 0:
            continue
        sl = slice(slot, slot + k)
        GLo[np.ix_(sec_l[s_i], np.arange(slot, slot + k))] = sec_V[s_i][:, :k]
        GRo[np.ix_(np.arange(slot, slot + k), sec_r[s_i])] = sec_W[s_i][:k, :]
        lam[sl] = info.sigma[s_i][:k]
        chg[sl] = info.sectors[s_i]
        slot += k
    st.Gamma[mode] = GLo
    st.Gamma[mode + 1] = GRo
    st.Lambda[mode] = lam
    st.charge[mode + 1] = chg
    return info


def apply_phases(st, phases):
    """Output phase screen e^{i phi_m n_m} on every mode (leaves photon statistics)."""
    d = st.d
    for m, ph in enumerate(phases):
        a = st.charge[m].astype(np.int64)
        b = st.charge[m + 1].astype(np.int64)
        dk = a[:, None, 0] - b[None, :, 0]
        db = a[:, None, 1] - b[None, :, 1]
        valid = (a[:, None, 0] < d) & (b[None, :, 0] < d)
        st.Gamma[m] *= np.where(valid, np.exp(1j * ph * (dk - db)), 1.0)
    return st


def _diag_mask(st, b):
    c = st.charge[b]
    return (c[:, 0] == c[:, 1]) & (c[:, 0] < st.d) & (bond_lambda(st, b) > 0)


def right_environments(st):
    """R[b] = partial trace of sites b..n-1, as a vector over bond b (diagonal charges)."""
    R = [None] * (st.n + 1)
    r = np.zeros(st.chi, dtype=np.complex128)
    r[_diag_mask(st, st.n)] = 1.0
    R[st.n] = r
    for b in range(st.n - 1, -1, -1):
        r = st.Gamma[b] @ R[b + 1]
        r = np.where(_diag_mask(st, b), r, 0.0)
        R[b] = r
    return R


def left_environments(st):
    """L[b] = partial trace of sites 0..b-1, as a vector over bond b."""
    L = [None] * (st.n + 1)
    l = np.where(_diag_mask(st, 0), 1.0 + 0j, 0.0)
    L[0] = l
    for b in range(st.n):
        l = L[b] @ st.Gamma[b]
        l = np.where(_diag_mask(st, b + 1), l, 0.0)
        L[b + 1] = l
    return L


def trace(st):
    """MPO trace (restates ``summary.Probability``, ``src/summary.py:11-26``)."""
    R = right_environments(st)
    return complex(np.sum(R[0]))


def marginals(st):
    """P[i, k] = probability of k photons in mode i (not normalised by the trace)."""
    d, chi = st.d, st.chi
    L = left_environments(st)
    R = right_environments(st)
    P = np.zeros((st.n, d), dtype=np.complex128)
    for i in range(st.n):
        a = st.charge[i, :, 0].astype(np.int64)
        b = st.charge[i + 1, :, 0].astype(np.int64)
        M = L[i][:, None] * st.Gamma[i] * R[i + 1][None, :]
        occ = a[:, None] - b[None, :]
        for k in range(d):
            P[i, k] = np.sum(M[occ == k])
    return P


def entanglement_entropy(st):
    """Per-bond entropy of normalised Lambda^2 (``src/summary.py:3-9``)."""
    out = np.zeros(st.n - 1)
    for i in range(st.n - 1):
        p = st.Lambda[i] ** 2
        tot = p.sum()
        if tot <= 0:
            continue
        p = p[p > 0] / tot
        out[i] = -np.sum(p * np.log2(p))
    return out


def bond_dims(st):
    return [int(np.sum(st.charge[b, :, 0] < st.d)) for b in range(st.n + 1)]
