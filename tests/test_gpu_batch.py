"""Independent circuits run side by side (engine.run_batch, the batched form at the host
level): every circuit computes exactly what it computes alone, on both SVD routes."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from bosonsampling_b200 import engine  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    torch.cuda.set_device(0)


@pytest.mark.parametrize("precision", ["fp64", "fp64-gram"])
def test_batch_equals_one_by_one(precision):
    specs = engine.batch_circuits(n_circuits=6, seed=77, chis=(16, 24, 32), d=3)
    for sp in specs:                       # keep the test small: 8-12 modes
        n = 8 + len(sp["photon_modes"]) % 5
        sp.update(n=n, photon_modes=list(range(0, n, 2)),
                  mesh=[b for b in sp["mesh"] if b[1] < n - 1 and b[0] < n], phases=sp["phases"][:n])
    seq = engine.run_batch(specs, concurrency=1, precision=precision, workers=2)
    par = engine.run_batch(specs, concurrency=4, precision=precision, workers=2)
    lpt = engine.run_batch(specs, concurrency=3, precision=precision, workers=2, largest_first=True)
    for (t1, p1), (t2, p2), (t3, p3) in zip(seq, par, lpt):   # results in input order
        assert t1 == t2 == t3
        assert np.array_equal(p1, p2) and np.array_equal(p1, p3)
        assert abs(t1) > 0
