"""The halo-exchange driver of one circuit over several ranks, on the CPU.

The schedule is checked by replaying it on versioned items (every update must see the
current version of each site and bond it reads; the root ends with every current
version), and the whole driver runs on two gloo ranks with the oracle's update standing
in for each rank's device state: the gathered state must equal the single-process
oracle run bit for bit."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from bosonsampling_b200 import halo, interferometer  # noqa: E402


def _replay(plan):
    """Replays the plan on versioned items, asserting that every read and the gather see current versions."""
    n, world = plan.n, plan.world
    current = {}
    store = [dict() for _ in range(world)]
    for l, (modes, _, _) in enumerate(plan.layers):
        for it, src, dst in plan.transfers[l]:
            assert src != dst
            assert store[src].get(it, 0) == current.get(it, 0), "sent a stale version"
            store[dst][it] = store[src].get(it, 0)
        for m in modes:
            r = plan.owner[m]
            for it in halo._reads(n, m):
                assert store[r].get(it, 0) == current.get(it, 0), f"layer {l} mode {m} reads a stale {it}"
        for m in modes:
            r = plan.owner[m]
            for it in halo._writes(m):
                current[it] = current.get(it, 0) + 1
                store[r][it] = current[it]
    for it, src, dst in plan.gather:
        assert store[src].get(it, 0) == current.get(it, 0)
        store[dst][it] = store[src].get(it, 0)
    for it, v in current.items():
        assert store[plan.root].get(it, 0) == v, f"root lacks {it}"


@pytest.mark.parametrize("n,world", [(6, 2), (8, 2), (9, 3), (16, 4), (12, 1), (5, 6)])
def test_plan_delivers_every_read_and_gathers_on_root(n, world):
    _, bs, _ = interferometer.circuit(n, 40 + n)
    plan = halo.HaloPlan(n, halo.layers_of(bs), world)
    _replay(plan)
    owner = plan.owner
    assert all(owner[i] <= owner[i + 1] for i in range(len(owner) - 1))   # contiguous blocks
    if world == 1:
        assert all(not tr for tr in plan.transfers) and not plan.gather


def test_other_root_and_custom_blocks():
    n = 10
    _, bs, _ = interferometer.circuit(n, 5)
    layers = halo.layers_of(bs)
    for owner, root in (([0, 0, 1, 1, 1, 2, 2, 2, 2], 2), ([1] * 4 + [0] * 5, 1), ([0] * 9, 0)):
        plan = halo.HaloPlan(n, layers, 3, owner=owner, root=root)
        _replay(plan)
        ran = [sum(len(plan.local_layer(l, r)[0]) for l in range(len(layers))) for r in range(3)]
        assert sum(ran) == len(bs)
    # everything on one rank of three: nothing moves but the gather to another root
    plan = halo.HaloPlan(n, layers, 3, owner=[0] * 9, root=2)
    assert all(not tr for tr in plan.transfers)
    assert plan.gather and all(src == 0 and dst == 2 for _, src, dst in plan.gather)


def test_brick_wall_exchange_is_one_site_and_one_bond_per_boundary():
    n, world, chi = 16, 4, 64
    _, bs, _ = interferometer.circuit(n, 7)
    plan = halo.HaloPlan(n, halo.layers_of(bs), world)
    boundaries = len(set(plan.owner)) - 1
    for l, tr in enumerate(plan.transfers):
        sites = [it for it, _, _ in tr if it[0] == halo.SITE]
        bonds = [it for it, _, _ in tr if it[0] == halo.BOND]
        assert len(sites) <= boundaries and len(bonds) <= boundaries, (l, tr)
        # every message crosses one block boundary only
        for it, src, dst in tr:
            assert abs(src - dst) == 1
    per_layer, gathered = plan.bytes_moved(chi)
    assert max(per_layer) <= boundaries * (chi * chi * 16 + chi * 16)


def test_balanced_blocks_and_bad_layers():
    layers = [([0, 2, 4, 6], [0.1] * 4, [0.2] * 4), ([1, 3, 5], [0.1] * 3, [0.2] * 3)]
    assert halo.block_owner(8, layers, 2) == [0, 0, 0, 1, 1, 1, 1]
    with pytest.raises(ValueError):
        halo.HaloPlan(8, [([0, 1], [0.1, 0.1], [0.0, 0.0])], 2)   # overlapping sites
    with pytest.raises(ValueError):
        halo.HaloPlan(8, [([7], [0.1], [0.0])], 2)                # mode out of range
    with pytest.raises(ValueError):
        halo.HaloPlan(8, layers, 2, owner=[0] * 6)                # wrong length
    # grouping by layer must not reorder beam splitters that share a site
    with pytest.raises(ValueError):
        halo.layers_of([(0, 0, 0.1, 0.0), (1, 1, 0.1, 0.0), (0, 2, 0.1, 0.0)])   # site 2: layer 1 then layer 0
    assert len(halo.layers_of([(0, 0, 0.1, 0.0), (1, 1, 0.1, 0.0), (0, 3, 0.1, 0.0)])) == 2   # site-disjoint: fine


class OracleSites:
    """Test stand-in for a rank's device state: the oracle's MPO and update on the host."""

    def __init__(self, st):
        from oracle import fock
        self.st, self.fock = st, fock

    def export(self, item):
        kind, i = item
        if kind == halo.SITE:
            return [torch.from_numpy(self.st.Gamma[i].copy())]
        return [torch.from_numpy(self.st.Lambda[i - 1].copy()), torch.from_numpy(self.st.charge[i].copy())]

    def buffers(self, item):
        chi = self.st.chi
        if item[0] == halo.SITE:
            return [torch.empty((chi, chi), dtype=torch.complex128)]
        return [torch.empty(chi, dtype=torch.float64), torch.empty((chi, 2), dtype=torch.int32)]

    def receive(self, item, tensors):
        kind, i = item
        if kind == halo.SITE:
            self.st.Gamma[i] = tensors[0].numpy()
        else:
            self.st.Lambda[i - 1] = tensors[0].numpy()
            self.st.charge[i] = tensors[1].numpy()

    def run(self, modes, thetas, phis):
        from oracle import mpo
        for m, th, ph in zip(modes, thetas, phis):
            mpo.bs_update(self.st, m, self.fock.update_tensor(interferometer.t_block(th, ph), self.st.d))

    def synchronize(self):
        pass


N, D, CHI, SEED = 7, 3, 10, 61


def _initial():
    from oracle import mpo
    st = mpo.initial_state(N, range(0, N, 2), 0.6, D, CHI)
    st.charge = st.charge.astype(np.int32)
    return st


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        _, bs, _ = interferometer.circuit(N, SEED)
        plan = halo.HaloPlan(N, halo.layers_of(bs), world)
        sites = OracleSites(_initial())
        halo.HaloCircuit(plan, {rank: sites}, halo.DistTransport(rank)).run()
        if rank == plan.root:
            out["state"] = (sites.st.Gamma.copy(), sites.st.Lambda.copy(), sites.st.charge.copy())
        out[f"ran{rank}"] = sum(len(plan.local_layer(l, rank)[0]) for l in range(len(plan.layers)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _single_process():
    from oracle import fock, mpo
    st = _initial()
    _, bs, _ = interferometer.circuit(N, SEED)
    for _, m, th, ph in bs:
        mpo.bs_update(st, m, fock.update_tensor(interferometer.t_block(th, ph), D))
    return st


def test_two_gloo_ranks_reproduce_the_single_process_circuit():
    world = 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    ref = _single_process()
    g, lam, chg = out["state"]
    assert out["ran0"] > 0 and out["ran1"] > 0            # both ranks did work
    np.testing.assert_array_equal(g, ref.Gamma)
    np.testing.assert_array_equal(lam, ref.Lambda)
    np.testing.assert_array_equal(chg, ref.charge)


def test_local_transport_reproduces_the_single_process_circuit():
    _, bs, _ = interferometer.circuit(N, SEED)
    plan = halo.HaloPlan(N, halo.layers_of(bs), 3)
    sites = {r: OracleSites(_initial()) for r in range(3)}
    halo.HaloCircuit(plan, sites, halo.LocalTransport()).run()
    ref = _single_process()
    np.testing.assert_array_equal(sites[0].st.Gamma, ref.Gamma)
    np.testing.assert_array_equal(sites[0].st.Lambda, ref.Lambda)
    np.testing.assert_array_equal(sites[0].st.charge, ref.charge)
