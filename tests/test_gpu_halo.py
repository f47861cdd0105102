"""One circuit partitioned over several handles with the halo exchange (the multi-rank
driver with its ranks emulated as handles of one process on one GPU, exchanging through
``bsmpo_get_site`` / ``bsmpo_put_site`` / ``bsmpo_get_bond`` / ``bsmpo_put_bond``): the
gathered state is exactly the single-handle run's."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from bosonsampling_b200 import _capi, engine, halo, interferometer  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    torch.cuda.set_device(0)


def _start(n, d, chi, precision, workers):
    sim = engine.MPOSimulator(n, d, chi)
    sim.set_precision(precision)
    sim.set_workers(workers)
    sim.init_single_photons(range(0, n, 2), 0.5)
    return sim


@pytest.mark.parametrize("n,d,chi,world,precision", [(10, 3, 24, 2, "fp64"), (10, 3, 24, 3, "fp64"),
                                                     (16, 4, 64, 4, "fp64-gram")])
def test_partitioned_circuit_equals_single_handle(n, d, chi, world, precision):
    _, bs, ph = interferometer.circuit(n, 70 + n)
    layers = halo.layers_of(bs)
    plan = halo.HaloPlan(n, layers, world)
    sims = [_start(n, d, chi, precision, 4) for _ in range(world)]
    ref = _start(n, d, chi, precision, 4)
    try:
        halo.HaloCircuit(plan, {r: halo.DeviceSites(s) for r, s in enumerate(sims)}, halo.LocalTransport()).run()
        ref.run_mesh([b[1] for b in bs], [b[2] for b in bs], [b[3] for b in bs])
        got, want = sims[plan.root].store(), ref.store()
        for a, b in zip(got, want):
            assert torch.equal(a, b)
        sims[plan.root].apply_phases(ph)
        ref.apply_phases(ph)
        (t1, p1), (t2, p2) = sims[plan.root].observables(), ref.observables()
        assert t1 == t2
        np.testing.assert_array_equal(p1, p2)
        assert sum(len(plan.local_layer(l, r)[0]) for l in range(len(layers)) for r in range(world)) == len(bs)
    finally:
        for s in sims + [ref]:
            s.close()


def test_site_and_bond_copies_round_trip_and_reject_bad_bonds():
    n, d, chi = 8, 3, 16
    _, bs, _ = interferometer.circuit(n, 3)
    with _start(n, d, chi, "fp64", 1) as a, _start(n, d, chi, "fp64", 1) as b:
        a.run_mesh([x[1] for x in bs[:10]], [x[2] for x in bs[:10]], [x[3] for x in bs[:10]])
        for s in range(n):
            b.put_site(s, a.get_site(s))
        for k in range(1, n):
            b.put_bond(k, *a.get_bond(k))
        for x, y in zip(a.store(), b.store()):
            assert torch.equal(x, y)
        assert a.trace() == b.trace()
        before = b.store()
        lam, chg = a.get_bond(3)
        bad = chg.flip(0).contiguous()            # occupied slots after empty ones / unsorted
        with pytest.raises(_capi.BsmpoError):
            b.put_bond(3, lam, bad)
        neg = lam.clone()
        neg[0] = -1.0                             # Lambda <= 0 on an occupied slot
        with pytest.raises(_capi.BsmpoError):
            b.put_bond(3, neg, chg)
        for x, y in zip(before, b.store()):       # a rejected bond leaves the state unchanged
            assert torch.equal(x, y)
        with pytest.raises(_capi.BsmpoError):
            b.put_bond(0, lam, chg)               # edge bonds are not exchanged
        with pytest.raises(_capi.BsmpoError):
            b.get_site(n, None)
