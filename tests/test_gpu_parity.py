"""GPU parity of libbsmpo against the CPU oracle (and the reference's own fixtures).

Tolerances: the plain path is FP64 end to end; singular values are compared
normwise per sector (|d sigma| <= 1e-10 sigma_max(sector)), observables relative to
the trace (|d P| <= 1e-10 trace).  Fixtures from the reference (complex64) are
compared at 1e-5.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from bosonsampling_b200 import _capi, engine, interferometer  # noqa: E402
from oracle import circuit, fock, mpo  # noqa: E402

TOL = 1e-10
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    torch.cuda.set_device(0)


def _spectra(lam, charge, d):
    out = {}
    for v, c in zip(lam, charge):
        if v > 0 and c[0] < d:
            out.setdefault((int(c[0]), int(c[1])), []).append(float(v))
    return {k: np.sort(np.array(v))[::-1] for k, v in out.items()}


def _close_spectra(a, b, atol):
    for key in set(a) | set(b):
        x, y = a.get(key, np.zeros(0)), b.get(key, np.zeros(0))
        n = max(len(x), len(y))
        np.testing.assert_allclose(np.pad(x, (0, n - len(x))), np.pad(y, (0, n - len(y))),
                                   rtol=0, atol=atol, err_msg=str(key))


# ------------------------------------------------------------------ Fock tensor
@pytest.mark.parametrize("d", [2, 3, 4, 5, 7])
def test_fock_tensor_matches_oracle(d):
    rng = np.random.default_rng(d)
    for _ in range(3):
        th, ph = rng.uniform(0, np.pi / 2), rng.uniform(0, 2 * np.pi)
        M = interferometer.t_block(th, ph)
        u = torch.empty(d ** 3, dtype=torch.complex128, device="cuda")
        m8 = engine._m8(M)
        _capi.check(_capi.lib().bsmpo_unitary(d, _capi.dptr(m8), ctypes.c_void_p(u.data_ptr()), None))
        torch.cuda.synchronize()
        np.testing.assert_allclose(u.cpu().numpy().reshape(d, d, d), fock.bs_tensor(M, d), atol=1e-14)


def test_fock_edges_exact():
    # r = 0 and t = 0: the reference's log-domain kernel needs a host branch; ours is exact
    d = 5
    for (t, r) in [(1.0, 0.0), (0.0, 1.0)]:
        ur = torch.empty(d ** 3, dtype=torch.float64, device="cuda")
        ui = torch.empty(d ** 3, dtype=torch.float64, device="cuda")
        _capi.check(_capi.lib().bsmpo_unitary_tr(d, t, 0.0, r, 0.0, ctypes.c_void_p(ur.data_ptr()),
                                                 ctypes.c_void_p(ui.data_ptr()), None))
        torch.cuda.synchronize()
        U = (ur + 1j * ui).cpu().numpy().reshape(d, d, d)
        ref = fock.bs_tensor(fock.tr_matrix(t, r), d)
        assert np.array_equal(U, ref), np.abs(U - ref).max()


def test_rand_u_matches_reference_tensors():
    """cuda_kernels.Rand_U draws the reference's phases (src/cuda_kernels.py:18-50)."""
    from bosonsampling_b200 import cuda_kernels
    fx = np.load(os.path.join(GOLDEN, "ref_bs_tensors.npz"))
    for key in fx.files:
        _, seed, d, r = key.split("_")
        seed, d, r = int(seed), int(d), float(r.replace("p", "."))
        # Rand_BS_MPS draws from RandomState(seed); Rand_U from the global RNG
        np.random.seed(seed)
        Ur, Ui = cuda_kernels.Rand_U(d, r)
        U = (Ur + 1j * Ui).cpu().numpy()
        ref = fock.tensor4_to_3(fx[key])
        if r != 0:   # the reference's r == 0 branch uses t = 1 without drawing its phase
            np.testing.assert_allclose(U, ref, atol=2e-6)


# ------------------------------------------------------------------ sector contraction drop-in
def test_update_mpo_dropin_matches_oracle_block_product():
    from bosonsampling_b200 import cuda_kernels
    n, d, chi = 8, 3, 24
    U, bs, ph = interferometer.circuit(n, 21)
    st = mpo.initial_state(n, range(0, n, 2), 0.6, d, chi)
    for (l, m, th, p) in bs[:9]:
        mpo.bs_update(st, m, fock.update_tensor(interferometer.t_block(th, p), d))
    mode = 3
    U3 = fock.update_tensor(interferometer.t_block(0.4, 1.1), d)
    CL, CC, CR = st.charge[mode], st.charge[mode + 1], st.charge[mode + 2]
    vl, vc, vr = [np.nonzero(c[:, 0] < d)[0] for c in (CL, CC, CR)]
    Glc = st.Gamma[mode][np.ix_(vl, vc)]
    Gcr = st.Gamma[mode + 1][np.ix_(vc, vr)]
    # change list of the centre charges (sorted)
    cc = CC[vc]
    chg_idx = [0] + [i for i in range(1, len(cc)) if tuple(cc[i]) != tuple(cc[i - 1])]
    chg = np.array([cc[i] for i in chg_idx], dtype=np.int32).T
    Ut = torch.from_numpy(U3.real.copy()).cuda(), torch.from_numpy(U3.imag.copy()).cuda()
    for cc0 in range(d):
        for cc1 in range(d):
            C = cuda_kernels.update_MPO(d, cc0, cc1, Ut[0], Ut[1], torch.from_numpy(Glc).cuda(),
                                        torch.from_numpy(Gcr).cuda(), torch.from_numpy(CL[vl]).cuda(),
                                        torch.from_numpy(CR[vr]).cuda(), chg, np.array(chg_idx, np.int32))
            C = C.cpu().numpy()
            # oracle: element-wise restatement of the kernel's sum (src/update_MPO_kernel.cu:440-455)
            ref = np.zeros_like(C)
            for i, a in enumerate(CL[vl]):
                for j, b in enumerate(CR[vr]):
                    if not (a[0] >= cc0 >= b[0] and a[1] >= cc1 >= b[1]):
                        continue
                    for c, q in enumerate(cc):
                        if a[0] >= q[0] >= b[0] and a[1] >= q[1] >= b[1]:
                            w = U3[a[0] - cc0, cc0 - b[0], a[0] - q[0]] * np.conj(U3[a[1] - cc1, cc1 - b[1], a[1] - q[1]])
                            ref[i, j] += w * Glc[i, c] * Gcr[c, j]
            scale = max(np.abs(ref).max(), 1e-300)
            np.testing.assert_allclose(C, ref, atol=1e-13 * scale)


@pytest.mark.parametrize("d,tau", [(3, 1), (4, 2), (5, 0), (5, 4)])
def test_update_mps_dropin_matches_elementwise_sum(d, tau):
    """The MPS variant (src/update_kernel.cu:193-769) against an element-wise
    restatement of its sum: T[l, r] = LL LR sum_c LC Glc Gcr U[cl - tau, tau - cr, cl - q]."""
    from bosonsampling_b200 import cuda_kernels
    rng = np.random.default_rng(10 * d + tau)
    len_l, len_c, len_r = 37, 29, 41
    CL = np.sort(rng.integers(0, d, len_l))[::-1].astype(np.int32)
    CC = np.sort(rng.integers(0, d, len_c)).astype(np.int32)
    CR = np.sort(rng.integers(0, d, len_r))[::-1].astype(np.int32)
    inc = np.full(d, -1, np.int32)
    for i, q in enumerate(CC):
        if inc[q] < 0:
            inc[q] = i
    Glc = rng.standard_normal((len_l, len_c)) + 1j * rng.standard_normal((len_l, len_c))
    Gcr = rng.standard_normal((len_c, len_r)) + 1j * rng.standard_normal((len_c, len_r))
    LL, LC, LR = (rng.uniform(0.1, 1.0, n) for n in (len_l, len_c, len_r))
    U3 = fock.update_tensor(interferometer.t_block(0.7, 0.3), d)
    Ut = torch.from_numpy(U3.real.copy()).cuda(), torch.from_numpy(U3.imag.copy()).cuda()
    T = cuda_kernels.update_MPS(d, tau, Ut[0], Ut[1], Glc, Gcr, LL, LC, LR, CL, CC, CR, inc).cpu().numpy()
    ref = np.zeros((len_l, len_r), dtype=np.complex128)
    for i, a in enumerate(CL):
        for j, b in enumerate(CR):
            if not (0 <= a - tau < d and 0 <= tau - b < d):
                continue
            for c, q in enumerate(CC):
                if a >= q >= b and a - q < d:
                    ref[i, j] += LC[c] * U3[a - tau, tau - b, a - q] * Glc[i, c] * Gcr[c, j]
            ref[i, j] *= LL[i] * LR[j]
    np.testing.assert_allclose(T, ref, atol=1e-13 * max(np.abs(ref).max(), 1e-300))


# ------------------------------------------------------------------ one BS update
@pytest.mark.parametrize("case", [(8, 3, 32, 5), (10, 4, 48, 12), (12, 5, 64, 20)])
def test_single_update_sigma_kept_and_weight(case):
    n, d, chi, nb = case
    U, bs, ph = interferometer.circuit(n, 100 + n)
    st = mpo.initial_state(n, range(0, n, 2), 0.5, d, chi)
    for (l, m, th, p) in bs[:nb]:
        mpo.bs_update(st, m, fock.update_tensor(interferometer.t_block(th, p), d))
    (l, m, th, p) = bs[nb]
    with engine.MPOSimulator(n, d, chi) as sim:
        sim.load_host(st.Gamma, st.Lambda, st.charge)
        S = interferometer.t_block(th, p)
        info_o = mpo.bs_update(st, m, fock.update_tensor(S, d))
        sim.bs_update(m, S)
        info_g = sim.last_update_info()
        tr, P = sim.observables()
    assert info_g["sectors"] == [tuple(x) for x in info_o.sectors]
    assert info_g["shape"] == [tuple(x) for x in info_o.shape]
    for sg, so in zip(info_g["sigma"], info_o.sigma):
        scale = max(float(so.max()) if len(so) else 0.0, 1e-300)
        np.testing.assert_allclose(sg, so, rtol=0, atol=TOL * scale)
    assert info_g["kept"] == list(info_o.kept)
    assert abs(info_g["trunc_weight"] - info_o.trunc_weight) <= TOL * max(
        sum(float(np.sum(s ** 2)) for s in info_o.sigma), 1e-300)
    tr_o = mpo.trace(st)
    assert abs(tr - tr_o) <= TOL * abs(tr_o)
    np.testing.assert_allclose(P, mpo.marginals(st), atol=TOL * abs(tr_o))


# ------------------------------------------------------------------ whole circuits
def _run_gpu(n, eta, d, chi, seed, phases=True, max_layers=None):
    """The mesh (or its first max_layers brick-wall layers) in one run_mesh call."""
    U, bs, ph = interferometer.circuit(n, seed)
    if max_layers is not None:
        bs = [b for b in bs if b[0] < max_layers]
    with engine.MPOSimulator(n, d, chi) as sim:
        sim.init_single_photons(range(0, n, 2), eta)
        sim.run_mesh([b[1] for b in bs], [b[2] for b in bs], [b[3] for b in bs])
        tw = sim.mesh_truncation()
        if phases:
            sim.apply_phases(ph)
        tr, P = sim.observables()
        g, lam, chg = sim.store()
        dims = sim.bond_dims()
    return tr, P, lam.cpu().numpy(), chg.cpu().numpy(), dims, tw


def _robust_dims(lam, chg, d, rel=1e-11):
    out = []
    for b in range(1, lam.shape[0] + 1):
        v = lam[b - 1] * (chg[b][:, 0] < d)
        out.append(int(np.sum(v > rel * max(v.max(), 1e-300))))
    return out


def _check_circuit(fx, w, tr, P, lam, chg, dims, tw):
    """Trace, marginals, per-bond spectra by charge, bond dimensions and per-update
    truncation weights against an oracle fixture (tolerances of the FP64 path)."""
    tr_o = complex(fx["trace"][0])
    assert abs(tr - tr_o) <= TOL * abs(tr_o), (tr, tr_o)
    np.testing.assert_allclose(P, fx["marginals"], atol=TOL * abs(tr_o))
    # bond dimensions counted over the singular values above 1e-11 of the bond's largest:
    # entries at the numerical-rank floor (~1e-13 of the largest) are rounding noise and
    # fall on either side of it in LAPACK and in the Jacobi rounds alike
    assert _robust_dims(lam, chg, w["d"]) == _robust_dims(fx["lam"], fx["charge"], w["d"])
    assert len(dims) == len(fx["bond_dims"])
    for b in range(1, w["n"]):
        _close_spectra(_spectra(lam[b - 1], chg[b], w["d"]), _spectra(fx["lam"][b - 1], fx["charge"][b], w["d"]),
                       TOL * max(1e-300, float(fx["lam"][b - 1].max())))
    # truncation weight of every update, normwise: |d tw| <= 1e-10 (total sigma^2 of the update)
    tw_o = fx["trunc_weight"]
    assert len(tw) == len(tw_o)
    bad = np.nonzero(np.abs(tw - tw_o) > TOL * fx["total_weight"])[0]
    assert len(bad) == 0, [(int(i), tw[i], tw_o[i]) for i in bad[:5]]


def test_plain_small_circuit_matches_oracle():
    """Workload 1: N=16, 8 photons (even modes), eta=0.5, d=4, chi=64, 120 BSs."""
    fx = np.load(os.path.join(GOLDEN, "oracle_plain_small.npz"))
    w = circuit.WORKLOADS["plain-small"]
    _check_circuit(fx, w, *_run_gpu(**w))


def test_plain_scale_circuit_matches_oracle():
    """Workload 2: N=32, 16 photons, eta=0.5, d=4, chi=256, 496 BSs (truncating)."""
    fx = np.load(os.path.join(GOLDEN, "oracle_plain_scale.npz"))
    w = circuit.WORKLOADS["plain-scale"]
    tr, P, lam, chg, dims, tw = _run_gpu(**w)
    _check_circuit(fx, w, tr, P, lam, chg, dims, tw)
    # size-independent property: every mode's marginal sums to the trace (positivity is
    # not one: truncating a density-matrix MPO can leave marginals slightly negative)
    np.testing.assert_allclose(P.sum(axis=1), np.full(w["n"], tr), atol=1e-12 * abs(tr))


def test_chi1024_workload_first_layers_match_oracle():
    """The benchmarked workload (N=64, 32 photons, eta=0.3, d=5, chi=1024, seed 1003):
    its first 11 brick-wall layers (341 updates; every interior bond saturated at
    chi = 1024 from layer 5 on) against the oracle's run of the same layers."""
    fx = np.load(os.path.join(GOLDEN, "oracle_precision_l11.npz"))
    w = circuit.WORKLOADS["precision"]
    tr, P, lam, chg, dims, tw = _run_gpu(**w, phases=False, max_layers=11)
    assert len(tw) == int(fx["n_bs"][0])
    _check_circuit(fx, w, tr, P, lam, chg, dims, tw)
    np.testing.assert_allclose(P.sum(axis=1), np.full(w["n"], tr), atol=1e-12 * abs(tr))


def test_concurrent_layers_match_one_by_one():
    """run_mesh runs a layer's beam splitters on several workers at once; every update
    computes exactly what it computes alone, so 1 and 4 workers agree bit for bit."""
    w = circuit.WORKLOADS["plain-small"]
    U, bs, ph = interferometer.circuit(w["n"], w["seed"])
    layers = {}
    for (l, m, th, p) in bs:
        layers.setdefault(l, []).append((m, th, p))
    out = []
    for workers in (1, 4):
        with engine.MPOSimulator(w["n"], w["d"], w["chi"]) as sim:
            sim.set_workers(workers)
            sim.init_single_photons(range(0, w["n"], 2), w["eta"])
            for l in sorted(layers):
                ops = layers[l]
                sim.run_mesh([o[0] for o in ops], [o[1] for o in ops], [o[2] for o in ops])
            info = sim.last_update_info()
            g, lam, chg = sim.store()
            out.append((g.cpu().numpy(), lam.cpu().numpy(), chg.cpu().numpy(), info["kept"]))
    (g1, l1, c1, k1), (g4, l4, c4, k4) = out
    assert np.array_equal(c1, c4) and k1 == k4
    assert np.array_equal(l1, l4)
    assert np.array_equal(g1, g4)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "ref_n*.npz"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_reference_fixtures_on_gpu(path):
    """The reference's own update sequence (its Rand_BS_MPS tensors) on the GPU path."""
    fx = np.load(path)
    n, n_in, d, chi = int(fx["n"]), int(fx["n_in"]), int(fx["d"]), int(fx["chi"])
    with engine.MPOSimulator(n, d, chi) as sim:
        sim.init_single_photons(range(n_in), 1.0 - float(fx["loss"]))
        tr0 = sim.trace()
        assert abs(tr0.real - float(fx["init_trace"])) < 1e-5
        for (mode, seed, r) in zip(fx["bs_mode"], fx["bs_seed"], fx["bs_refl"]):
            U3 = fock.reference_random_tensor(int(seed), d, float(r))
            sim.bs_update_tensor(int(mode), torch.from_numpy(U3.reshape(-1)).cuda())
        tr, P = sim.observables()
    assert abs(tr.real - float(fx["final_trace"])) < 1e-5
    np.testing.assert_allclose(P.real, fx["final_marginals"], atol=1e-5)


# ------------------------------------------------------------------ known answers on the GPU
def test_kat_single_photon_marginals():
    n, eta = 6, 0.8
    U, bs, ph = interferometer.circuit(n, 7)
    for j in (0, 3):
        with engine.MPOSimulator(n, 2, 8) as sim:
            sim.init_single_photons([j], eta)
            for (l, m, th, p) in bs:
                sim.bs_update(m, interferometer.t_block(th, p))
            tr, P = sim.observables()
        np.testing.assert_allclose(P[:, 1].real, eta * np.abs(U[:, j]) ** 2, atol=1e-13)
        assert abs(tr - 1.0) < 1e-13


def test_kat_trace_is_binomial_cdf():
    from scipy.stats import binom
    for (n, eta, d) in [(16, 0.5, 4), (10, 0.3, 5)]:
        with engine.MPOSimulator(n, d, 64) as sim:
            sim.init_single_photons(range(0, n, 2), eta)
            tr = sim.trace()
        assert abs(tr.real - binom.cdf(d - 1, len(range(0, n, 2)), eta)) < 1e-13


def test_kat_hong_ou_mandel():
    with engine.MPOSimulator(2, 3, 9) as sim:
        sim.init_single_photons([0, 1], 1.0)
        sim.bs_update(0, interferometer.t_block(np.pi / 4, 0.0))
        tr, P = sim.observables()
    assert abs(P[0, 1]) < 1e-15
    np.testing.assert_allclose(P[0].real, [0.5, 0.0, 0.5], atol=1e-14)


# ------------------------------------------------------------------ initial state on the device
@pytest.mark.parametrize("n,d,chi,tp", [(6, 3, 16, None), (16, 4, 64, None), (9, 5, 32, None), (6, 4, 16, 2)])
def test_product_state_built_on_device_matches_oracle(n, d, chi, tp):
    rhos = [mpo.single_photon_rho(d, 0.4) if i % 2 == 0 else mpo.vacuum_rho(d) for i in range(n)]
    rng = np.random.default_rng(n * d)
    # one mode with a coherence (off-diagonal) entry, so ket != bra charges occur
    rhos[1] = rhos[1].copy()
    rhos[1][0, 1] = rhos[1][1, 0] = 0.1 + 0.05j * rng.standard_normal()
    rhos[1][1, 0] = np.conj(rhos[1][0, 1])
    rhos[1][1, 1] = 0.3
    st = mpo.product_state(n, rhos, d, chi, total_photons=tp)
    with engine.MPOSimulator(n, d, chi) as sim:
        sim.init_product(rhos, total_photons=tp, canonicalize=False)
        g, lam, chg = sim.store()
        dims = sim.bond_dims()
    np.testing.assert_array_equal(chg.cpu().numpy(), st.charge)
    np.testing.assert_array_equal(lam.cpu().numpy(), st.Lambda)
    np.testing.assert_array_equal(g.cpu().numpy(), st.Gamma)
    assert dims == mpo.bond_dims(st)


def test_init_product_rejects_small_chi():
    # bond 0 lists the four diagonal totals (c, c), c < 4: three slots are too few
    with engine.MPOSimulator(8, 4, 3) as sim:
        with pytest.raises(_capi.BsmpoError, match="smaller than the product-state"):
            sim.init_single_photons(range(0, 8, 2), 0.5)


# ------------------------------------------------------------------ drop-ins and errors
def test_initialize_dropin_matches_oracle():
    from bosonsampling_b200 import MPO
    for (n, n_in, d, loss) in [(6, 3, 3, 0.3), (8, 4, 4, 0.5)]:
        G, L, C = MPO.Initialize("Single photon", n, n_in, None, d, {"loss": loss})
        st = mpo.initial_state(n, range(n_in), 1 - loss, d, d * d)
        for b in range(1, n):
            _close_spectra(_spectra(L[b - 1], C[b], d), _spectra(st.Lambda[b - 1], st.charge[b], d), 1e-12)


def test_probability_dropin_and_worker():
    from bosonsampling_b200 import gpu_algorithm, summary
    n, d, chi = 8, 3, 32
    st = mpo.initial_state(n, range(4), 0.7, d, chi)
    tr = summary.Probability(n, d, st.Gamma, st.Lambda, st.charge)
    assert abs(tr - mpo.trace(st)) < 1e-13
    wk = gpu_algorithm.Worker()
    wk.ExperimentInit("Single photon", n, 4, None, d, chi, {"loss": 0.3}, seed=5)
    ok, prob, EE, _ = wk.Simulate()
    assert ok and prob.shape == (n + 1,) and EE.shape == (n - 1, n + 1)
    # oracle: same mesh, same input, trace after the last layer
    U, bs, ph = interferometer.circuit(n, 5)
    for (l, m, th, p) in bs:
        mpo.bs_update(st, m, fock.update_tensor(interferometer.t_block(th, p), d))
    assert abs(prob[-1] - mpo.trace(st).real) < 1e-6


def test_errors_are_reported_not_raised_across_the_abi():
    L = _capi.lib()
    h = ctypes.c_void_p()
    assert L.bsmpo_create(1, 4, 16, 0, ctypes.byref(h)) == -1          # n < 2
    assert b"create" in L.bsmpo_last_error(None)
    _capi.check(L.bsmpo_create(4, 3, 8, 0, ctypes.byref(h)))
    S = engine._m8(np.eye(2))
    assert L.bsmpo_bs_update(h, 0, _capi.dptr(S)) == -1              # no state loaded
    st = mpo.product_state(4, [mpo.single_photon_rho(3, 0.5)] + [mpo.vacuum_rho(3)] * 3, 3, 8)
    g, l, c = st.Gamma, st.Lambda, st.charge.copy()
    c[0, [0, 1]] = c[0, [1, 0]]                                        # bond 0 no longer sorted
    gd, ld, cd = (torch.from_numpy(x).cuda() for x in (g, l, c))
    rc = L.bsmpo_load_state(h, ctypes.c_void_p(gd.data_ptr()), ctypes.c_void_p(ld.data_ptr()),
                            ctypes.c_void_p(cd.data_ptr()))
    assert rc == -1 and b"sorted" in L.bsmpo_last_error(h)
    L.bsmpo_destroy(h)
