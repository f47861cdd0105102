"""A mesh over a host-resident state (bsmpo_run_mesh_host): the site copies overlap the
updates, and the result is exactly that of load + run_mesh + store."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from bosonsampling_b200 import _capi, engine, interferometer  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    torch.cuda.set_device(0)


def _layers(n, seed):
    _, bs, _ = interferometer.circuit(n, seed)
    layers = [[] for _ in range(n)]
    for (l, m, th, p) in bs:
        layers[l].append((m, th, p))
    return layers


def _ops(layers, first, count):
    o = [x for L in range(first, first + count) for x in layers[L]]
    return [x[0] for x in o], [x[1] for x in o], [x[2] for x in o]


def _host(state):
    return tuple(x.cpu().pin_memory() for x in state)


@pytest.mark.parametrize("precision,workers", [("fp64", 1), ("fp64", 4), ("fp64-gram", 4)])
def test_host_mesh_equals_device_mesh(precision, workers):
    n, d, chi = 10, 3, 24
    layers = _layers(n, 5)
    with engine.MPOSimulator(n, d, chi) as sim:
        sim.set_precision(precision)
        sim.set_workers(workers)
        sim.init_single_photons(range(0, n, 2), 0.5)
        sim.run_mesh(*_ops(layers, 0, 3))
        start = sim.store()
        host_in = _host(start)
        # reference: device-resident state
        sim.load(*start)
        sim.run_mesh(*_ops(layers, 3, 2))
        ref = [x.cpu() for x in sim.store()]
        tr_ref = sim.trace()
        # host-resident: into separate outputs, then in place
        out = sim.run_mesh_host(*_ops(layers, 3, 2), host_in)
        for a, b in zip(out, ref):
            assert torch.equal(a, b)
        assert sim.trace() == tr_ref
        inplace = tuple(x.clone().pin_memory() for x in host_in)
        sim.run_mesh_host(*_ops(layers, 3, 2), inplace, inplace)
        for a, b in zip(inplace, ref):
            assert torch.equal(a, b)
        # the input is untouched when the outputs are separate
        for a, b in zip(host_in, start):
            assert torch.equal(a, b.cpu())


def test_host_mesh_empty_and_unpinned():
    n, d, chi = 8, 3, 16
    with engine.MPOSimulator(n, d, chi) as sim:
        sim.init_single_photons(range(0, n, 2), 0.5)
        start = [x.cpu() for x in sim.store()]          # pageable host memory
        out = sim.run_mesh_host([], [], [], start)      # no updates: a round trip
        for a, b in zip(out, start):
            assert torch.equal(a, b)
        layers = _layers(n, 9)
        ref_sim_state = sim.run_mesh_host(*_ops(layers, 0, 2), start)
        sim.load(*[x.cuda() for x in start])
        sim.run_mesh(*_ops(layers, 0, 2))
        for a, b in zip(ref_sim_state, sim.store()):
            assert torch.equal(a, b.cpu())


def test_host_mesh_rejects_a_bad_state():
    n, d, chi = 8, 3, 16
    with engine.MPOSimulator(n, d, chi) as sim:
        sim.init_single_photons(range(0, n, 2), 0.5)
        g, lam, c = [x.cpu() for x in sim.store()]
        bad = c.clone()
        bad[3, 0] = torch.tensor([d + 1, 0], dtype=torch.int32)   # charge out of range
        with pytest.raises(_capi.BsmpoError, match="bond 3"):
            sim.run_mesh_host([0], [0.3], [0.1], (g, lam, bad))
        with pytest.raises(_capi.BsmpoError, match="no state loaded"):
            sim.run_mesh([0], [0.3], [0.1])
