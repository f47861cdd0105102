"""Generate the golden fixtures that pin the CPU oracle to the reference simulator.

Run in the build container (it reads the reference checkout; nothing at test time
does):

    python tests/golden/make_golden.py /path/to/reference

It imports the reference's own CPU algorithm, ``src/MPO.py`` (``Rand_BS_MPS``,
``Initialize``, ``InitializationMPO.Update``) and ``src/summary.py``
(``Probability``, ``EntanglementEntropy``), with two adjustments made in memory only:

* ``qutip`` is replaced by a stub module (it is only used for Gaussian inputs,
  ``src/MPO.py:2,34-40``, which no fixture uses);
* the scatter loop's sector index ``tau = i * d + j`` (``src/MPO.py:288``) is replaced
  by the loop position, which is what that line means when the centre-charge ranges
  are not the full ``0..d-1``.

The reference computes in complex64, so fixtures are compared at 1e-5 relative.
Cases avoid truncation cuts that split a degenerate ket/bra-swapped sector pair
(where the reference's choice is arbitrary); the generator asserts that no such split
happened in the recorded cases.
"""
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def load_reference(ref_root):
    stub = types.ModuleType("qutip")
    stub.squeeze = lambda *a, **k: None
    stub.thermal_dm = lambda *a, **k: None
    sys.modules.setdefault("qutip", stub)
    src = open(os.path.join(ref_root, "src", "MPO.py")).read()
    old = "tau = i * d + j"
    assert src.count(old) == 1
    src = src.replace(old, "tau = (i - smallest_cr_0) * (largest_cl_1 - smallest_cr_1 + 1) + (j - smallest_cr_1)")
    mpo_mod = types.ModuleType("ref_MPO")
    exec(compile(src, "ref_MPO.py", "exec"), mpo_mod.__dict__)
    summ = types.ModuleType("ref_summary")
    exec(compile(open(os.path.join(ref_root, "src", "summary.py")).read(), "ref_summary.py", "exec"),
         summ.__dict__)
    return mpo_mod, summ


class SvdRecorder:
    """Wraps numpy.linalg.svd to record each sector's singular values in call order."""

    def __init__(self):
        self.calls = []
        self._orig = np.linalg.svd

    def __enter__(self):
        def rec(a, *args, **kw):
            out = self._orig(a, *args, **kw)
            self.calls.append((a.shape, np.asarray(out[1], dtype=np.float64).copy()))
            return out
        np.linalg.svd = rec
        return self

    def __exit__(self, *exc):
        np.linalg.svd = self._orig


def embed(Gamma, Lambda, charge, chi, d):
    """Reference Initialize output ([n,c,c],[n-1,c],[n+1,c,2]) -> its internal layout at chi."""
    n, c, _ = Gamma.shape
    G = np.zeros((chi, chi, n), dtype=np.complex64)
    L = np.zeros((chi, n - 1), dtype=np.float32)
    C = np.full((chi, n + 1, 2), d, dtype=np.int32)
    G[:c, :c, :] = np.transpose(Gamma, (1, 2, 0))
    L[:c, :] = np.transpose(Lambda, (1, 0))
    C[:c, :, :] = np.transpose(charge, (1, 0, 2))
    # empty internal slots: the CPU update masks by Lambda > 0; edges need a charge that
    # matches no valid block
    return G, L, C


def swap_symmetric(charges, lam, d):
    valid = (lam > 0) & (charges[:, 0] < d)
    from collections import Counter
    cnt = Counter(map(tuple, charges[valid].tolist()))
    return all(cnt[(a, b)] == cnt[(b, a)] for (a, b) in cnt)


def run_case(ref, summ, name, n, n_in, d, loss, chi, bs_seq):
    """Initialize + a sequence of reference Updates; returns a fixture dict."""
    Gamma, Lambda, charge = ref.Initialize("Single photon", n, n_in, None, d, {"loss": loss})
    out = {"n": n, "n_in": n_in, "d": d, "loss": loss, "chi": chi}
    out["init_lambda"] = np.asarray(Lambda, dtype=np.float64)
    out["init_charge"] = np.asarray(charge)
    out["init_trace"] = float(np.real(summ.Probability(n, d, Gamma, Lambda, charge)))
    G, L, C = embed(Gamma, Lambda, charge, chi, d)
    obj = object.__new__(ref.InitializationMPO)
    obj.n_modes, obj.local_hilbert_space_dimension, obj.bond_dimension = n, d, chi
    obj.Gamma, obj.Lambda, obj.charge = G, L, C
    obj.edge_Lambda = np.ones(chi, dtype="float32")
    modes, seeds, refl = [], [], []
    sig_flat, sig_len, sig_shape = [], [], []
    sec_ids = []
    for (mode, seed, r) in bs_seq:
        sec_ids.extend(nonempty_sectors(obj, mode, d, n, chi))
        obj.Unitary = ref.Rand_BS_MPS(seed, d, r)
        with SvdRecorder() as rec:
            obj.Update(mode)
        assert swap_symmetric(obj.charge[:, mode + 1, :], obj.Lambda[:, mode], d), \
            "reference truncation split a swapped pair in %s" % name
        modes.append(mode); seeds.append(seed); refl.append(r)
        sig_len.append(len(rec.calls))
        for (shape, s) in rec.calls:
            sig_shape.append(shape)
            sig_flat.append(s)
    out["bs_mode"] = np.array(modes, dtype=np.int32)
    out["bs_seed"] = np.array(seeds, dtype=np.int64)
    out["bs_refl"] = np.array(refl, dtype=np.float64)
    out["sectors_per_bs"] = np.array(sig_len, dtype=np.int32)
    out["sector_shape"] = np.array(sig_shape, dtype=np.int32).reshape(-1, 2)
    out["sector_id"] = np.array(sec_ids, dtype=np.int32).reshape(-1, 2)
    assert len(sec_ids) == len(sig_shape), name
    out["sigma_len"] = np.array([len(s) for s in sig_flat], dtype=np.int32)
    out["sigma"] = np.concatenate(sig_flat) if sig_flat else np.zeros(0)
    # final state back in [site, chi, chi] layout
    Gf = np.transpose(obj.Gamma, (2, 0, 1)).astype(np.complex128)
    Lf = np.transpose(obj.Lambda, (1, 0)).astype(np.float64)
    Cf = np.transpose(obj.charge, (1, 0, 2))
    out["final_lambda"] = Lf
    out["final_charge"] = Cf
    out["final_trace"] = float(np.real(summ.Probability(n, d, Gf, Lf, Cf)))
    out["final_ee"] = np.asarray(summ.EntanglementEntropy(Lf), dtype=np.float64)
    # marginals of the reference's final state: independent contraction written here
    out["final_marginals"] = marginals_from_arrays(Gf, Lf, Cf, d)
    return out


def nonempty_sectors(obj, mode, d, n, chi):
    """Centre charges the reference's update loop visits with non-empty L and R sets.

    Same masks as ``src/MPO.py:182-206`` (charge blocks with Lambda > 0), evaluated on
    the reference object's own arrays; used only to label the recorded SVD calls.
    """
    edge = np.ones(chi)
    LL = edge if mode == 0 else obj.Lambda[:, mode - 1]
    LR = edge if mode == n - 2 else obj.Lambda[:, mode + 1]
    CL, CR = obj.charge[:, mode], obj.charge[:, mode + 2]
    vl = (LL > 0) & (CL[:, 0] < d) & (CL[:, 1] < d)
    vr = (LR > 0) & (CR[:, 0] < d) & (CR[:, 1] < d)
    hi0 = int(CL[CL[:, 0] != d, 0].max()) if (CL[:, 0] != d).any() else 0
    hi1 = int(CL[CL[:, 1] != d, 1].max()) if (CL[:, 1] != d).any() else 0
    lo0, lo1 = int(CR[:, 0].min()), int(CR[:, 1].min())
    out = []
    for c0 in range(lo0, hi0 + 1):
        for c1 in range(lo1, hi1 + 1):
            nl = np.sum(vl & (CL[:, 0] >= c0) & (CL[:, 1] >= c1))
            nr = np.sum(vr & (CR[:, 0] <= c0) & (CR[:, 1] <= c1))
            if nl and nr:
                out.append((c0, c1))
    return out


def marginals_from_arrays(G, L, C, d):
    """P[i, k] from raw arrays: sum over charge-diagonal paths with occupation k at site i."""
    n, chi, _ = G.shape
    lam = [np.ones(chi)] + [L[i] for i in range(n - 1)] + [np.ones(chi)]
    diag = [(C[b, :, 0] == C[b, :, 1]) & (lam[b] > 0) & (C[b, :, 0] < d) for b in range(n + 1)]
    R = [None] * (n + 1)
    R[n] = diag[n].astype(np.complex128)
    for b in range(n - 1, -1, -1):
        R[b] = np.where(diag[b], G[b] @ R[b + 1], 0)
    Lv = [None] * (n + 1)
    Lv[0] = diag[0].astype(np.complex128)
    for b in range(n):
        Lv[b + 1] = np.where(diag[b + 1], Lv[b] @ G[b], 0)
    P = np.zeros((n, d))
    for i in range(n):
        occ = C[i, :, 0][:, None].astype(int) - C[i + 1, :, 0][None, :].astype(int)
        M = (Lv[i][:, None] * G[i] * R[i + 1][None, :]).real
        for k in range(d):
            P[i, k] = M[occ == k].sum()
    return P


def brick_wall(n, layers, seed0, rng):
    seq = []
    s = seed0
    for layer in range(layers):
        for mode in range(layer % 2, n - 1, 2):
            seq.append((mode, s, float(rng.uniform(0.2, 0.95))))
            s += 1
    return seq


def main(ref_root):
    ref, summ = load_reference(ref_root)
    rng = np.random.default_rng(20261203)
    cases = {
        # no truncation: chi large enough for the exact state
        "ref_n6_d3": dict(n=6, n_in=3, d=3, loss=0.3, chi=64, layers=6),
        "ref_n8_d4": dict(n=8, n_in=4, d=4, loss=0.5, chi=128, layers=5),
        "ref_n5_d5": dict(n=5, n_in=3, d=5, loss=0.2, chi=128, layers=5),
        # truncating case (checked: no split of a swapped pair)
        "ref_n8_d3_trunc": dict(n=8, n_in=4, d=3, loss=0.4, chi=list(range(12, 40)), layers=6),
    }
    for name, c in cases.items():
        seq = brick_wall(c["n"], c["layers"], 100, rng)
        fx = None
        for chi in (c["chi"] if isinstance(c["chi"], list) else [c["chi"]]):
            try:
                fx = run_case(ref, summ, name, c["n"], c["n_in"], c["d"], c["loss"], chi, seq)
            except AssertionError:
                continue
            if isinstance(c["chi"], list):
                # a truncating case must actually truncate
                full = run_case(ref, summ, name, c["n"], c["n_in"], c["d"], c["loss"], 256, seq)
                if np.allclose(np.sort(full["final_lambda"], axis=1)[:, -chi:], np.sort(fx["final_lambda"], axis=1)[:, -chi:]):
                    fx = None
                    continue
            break
        assert fx is not None, name
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **fx)
        print(name, "chi", fx["chi"], "bs", len(seq), "trace", fx["init_trace"], "->", fx["final_trace"],
              "bytes", os.path.getsize(path))
    # the reference's own beam-splitter tensors (src/MPO.py:6-18)
    tens = {}
    for (seed, d, r) in [(0, 4, 0.0), (7, 4, 0.5), (11, 5, 0.3), (3, 3, 0.9), (5, 5, 1.0)]:
        tens["U_%d_%d_%s" % (seed, d, str(r).replace(".", "p"))] = ref.Rand_BS_MPS(seed, d, r).astype(np.complex128)
    np.savez_compressed(os.path.join(HERE, "ref_bs_tensors.npz"), **tens)
    print("tensors", list(tens))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
