"""The library's update against the reference's own update at the benchmarked size.

N = 64, d = 5, chi = 1024 with every bond full: four layer-6 updates of the bench
workload, which ``tests/golden/make_ref_chi1024.py`` ran through the reference's
``InitializationMPO.Update`` (complex64) from the oracle's state.  Here the library
starts from the same oracle state and runs the same updates on the plain FP64 path
(the Gram route is held to the plain path's marginals and truncation weights at this
size by ``test_gpu_mixed.py`` and by the bench's error columns).  Its
new centre-bond spectra must agree with the reference's per charge at 1e-5 of the
largest value (the reference's precision).  Where the reference's cut split a
ket/bra-swapped pair (it keeps an arbitrary member, the library neither), the reference
holds that one extra value."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from bosonsampling_b200 import engine, interferometer  # noqa: E402
from test_oracle_golden import TOL, _bond_spectrum  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def start():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    torch.cuda.set_device(0)
    import sys
    sys.path.insert(0, GOLDEN)
    from make_ref_chi1024 import oracle_start
    return oracle_start()


@pytest.mark.parametrize("precision", ["fp64"])
def test_library_update_matches_reference_at_chi1024(start, precision):
    st, timed = start
    fx = np.load(os.path.join(GOLDEN, "ref_chi1024_layer6.npz"))
    d = int(fx["d"])
    assert [m for m, _, _ in timed] == fx["mode"].tolist()
    with engine.MPOSimulator(st.n, st.d, st.chi) as sim:
        sim.set_precision(precision)
        sim.load_host(st.Gamma, st.Lambda, st.charge)
        for i, (m, th, ph) in enumerate(timed):
            sim.bs_update(m, interferometer.t_block(th, ph))
            lam, chg = sim.get_bond(m + 1)
            ours = _bond_spectrum(lam.cpu().numpy(), chg.cpu().numpy(), d)
            ref = _bond_spectrum(fx["ref_lambda"][i], fx["ref_charge"][i], d)
            scale = max(v.max() for v in ours.values())
            keys = set(ours) | set(ref)
            longer = [k for k in keys if len(ref.get(k, ())) != len(ours.get(k, ()))]
            if fx["ref_split_pair"][i]:
                assert len(longer) == 1 and len(ref[longer[0]]) == len(ours.get(longer[0], ())) + 1
            else:
                assert not longer
            for k in keys:
                x, y = ours.get(k, np.zeros(0)), ref.get(k, np.zeros(0))
                n = min(len(x), len(y))
                np.testing.assert_allclose(x[:n], y[:n], rtol=0, atol=TOL * scale, err_msg=f"{precision} {m} {k}")
