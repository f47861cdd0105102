"""GPU parity of the Gram / Hermitian-eigen route of the sector SVD (precision mode
'fp64-gram': FP64 contractions, FP64 Gram matrix, Householder tridiagonalisation,
bisection and inverse iteration) against the CPU oracle.

The route drops singular values below about 2e-6 of each sector's largest as zero,
so bond dimensions may differ from the plain path's in the first, untruncated
layers; everything of weight agrees.  Tolerances (written here): singular values
above 1e-5 of their sector's largest within 1e-9 of the largest; trace and every
marginal within 1e-8 of the trace; per-update truncation weight within 1e-8 of the
update's total weight.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from bosonsampling_b200 import engine, interferometer  # noqa: E402
from oracle import circuit, fock, mpo  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SIG_TOL = 1e-9
OBS_TOL = 1e-8


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    torch.cuda.set_device(0)


@pytest.mark.parametrize("case", [(8, 3, 32, 5), (10, 4, 48, 12), (12, 5, 64, 20), (12, 4, 24, 30)])
def test_gram_single_update_sigma(case):
    n, d, chi, nb = case
    U, bs, ph = interferometer.circuit(n, 100 + n)
    st = mpo.initial_state(n, range(0, n, 2), 0.5, d, chi)
    for (l, m, th, p) in bs[:nb]:
        mpo.bs_update(st, m, fock.update_tensor(interferometer.t_block(th, p), d))
    (l, m, th, p) = bs[nb]
    with engine.MPOSimulator(n, d, chi) as sim:
        sim.set_precision("fp64-gram")
        sim.load_host(st.Gamma, st.Lambda, st.charge)
        S = interferometer.t_block(th, p)
        info_o = mpo.bs_update(st, m, fock.update_tensor(S, d))
        sim.bs_update(m, S)
        info_g = sim.last_update_info()
        tr, P = sim.observables()
    assert info_g["sectors"] == [tuple(x) for x in info_o.sectors]
    assert info_g["shape"] == [tuple(x) for x in info_o.shape]
    for sg, so in zip(info_g["sigma"], info_o.sigma):
        if len(so) == 0:
            continue
        smax = float(so.max())
        big = so > 1e-5 * smax
        np.testing.assert_allclose(sg[big], so[big], rtol=0, atol=SIG_TOL * smax)
        assert np.all(sg[~big] <= 2e-5 * smax)
    tr_o = mpo.trace(st)
    assert abs(tr - tr_o) <= OBS_TOL * abs(tr_o)
    np.testing.assert_allclose(P, mpo.marginals(st), atol=OBS_TOL * abs(tr_o))


def _run(w, precision, max_layers=None, phases=True, workers=None):
    U, bs, ph = interferometer.circuit(w["n"], w["seed"])
    if max_layers is not None:
        bs = [b for b in bs if b[0] < max_layers]
    with engine.MPOSimulator(w["n"], w["d"], w["chi"]) as sim:
        sim.set_precision(precision)
        if workers:
            sim.set_workers(workers)
        sim.init_single_photons(range(0, w["n"], 2), w["eta"])
        sim.run_mesh([b[1] for b in bs], [b[2] for b in bs], [b[3] for b in bs])
        tw = sim.mesh_truncation()
        if phases:
            sim.apply_phases(ph)
        tr, P = sim.observables()
        g, lam, chg = sim.store()
    return tr, P, tw, g.cpu().numpy(), lam.cpu().numpy(), chg.cpu().numpy()


@pytest.mark.parametrize("name,fixture,layers", [
    ("plain-small", "oracle_plain_small.npz", None),
    ("plain-scale", "oracle_plain_scale.npz", None),
    ("precision", "oracle_precision_l11.npz", 11),
])
def test_gram_circuit_matches_oracle(name, fixture, layers):
    fx = np.load(os.path.join(GOLDEN, fixture))
    w = circuit.WORKLOADS[name]
    tr, P, tw, _, _, _ = _run(w, "fp64-gram", max_layers=layers, phases=layers is None)
    tr_o = complex(fx["trace"][0])
    assert abs(tr - tr_o) <= OBS_TOL * abs(tr_o), (tr, tr_o)
    err = np.abs(P - fx["marginals"]).max() / abs(tr_o)
    assert err <= OBS_TOL, err
    tw_o = fx["trunc_weight"]
    assert len(tw) == len(tw_o)
    assert np.all(np.abs(tw - tw_o) <= OBS_TOL * fx["total_weight"] + 1e-300)


def test_gram_concurrent_layers_match_one_by_one():
    w = circuit.WORKLOADS["plain-small"]
    a = _run(w, "fp64-gram", workers=1)
    b = _run(w, "fp64-gram", workers=4)
    for x, y in zip(a[3:], b[3:]):
        assert np.array_equal(x, y)
