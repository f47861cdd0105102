"""One circuit over several ranks: contiguous blocks of modes per rank, and a halo
exchange of boundary sites between the layers of a brick-wall mesh.

The reference spreads one layer's beam splitters over its GPU ranks by shipping each
request's two sites to a free rank and back (``src/beam_splitter_parallel/Full.py:149-166``
with ``Rank.py:32-206``), and places sites on nodes round-robin
(``src/fully_parallel/Full.py:70-103``).  Here every rank keeps the whole chain's layout
resident in its own HBM (the initial state is built identically on every rank, so it
starts replicated), runs the beam splitters whose left mode lies in its block, and before
each layer receives exactly the sites and bonds its updates read whose current version
another rank wrote.  In a brick-wall layer that is, per block boundary, one site's Gamma
(chi^2 complex128) and one bond's Lambda and charges, sent in the direction the layer's
parity gives; nothing else crosses between ranks until the final gather.

The schedule (``HaloPlan``) is computed from the mesh alone, identically on every rank,
so the sends and receives of a layer pair up without any negotiation.  The transport is
``torch.distributed`` point-to-point (NCCL between GPUs: one message per site or bond
array, received into local HBM and copied into the handle's state by
``bsmpo_put_site`` / ``bsmpo_put_bond``), or, for several handles driven by one process,
direct device copies (``LocalTransport``).
"""
from collections import defaultdict

import numpy as np

SITE, BOND = "site", "bond"


def _reads(n, m):
    """Items the update on modes (m, m+1) reads: its two sites and bonds m, m+1, m+2
    (the bond Lambda / charges on the left, centre and right; the edge bonds 0 and n
    never change and are not exchanged)."""
    return [(SITE, m), (SITE, m + 1)] + [(BOND, b) for b in (m, m + 1, m + 2) if 1 <= b <= n - 1]


def _writes(m):
    """Items the update on modes (m, m+1) writes: its two sites and the centre bond."""
    return [(SITE, m), (SITE, m + 1), (BOND, m + 1)]


def layers_of(mesh):
    """Group a mesh ``[(layer, mode, theta, phi), ...]`` into layers in order of first
    appearance: ``[(modes, thetas, phis), ...]``.  Raises ValueError where the grouping
    would move a beam splitter before an earlier one on a shared site (the grouped
    circuit would differ from the mesh applied in its order)."""
    order, groups, pos, last = [], defaultdict(list), {}, {}
    for layer, mode, th, ph in mesh:
        if layer not in groups:
            pos[layer] = len(order)
            order.append(layer)
        g = pos[layer]
        for site in (int(mode), int(mode) + 1):
            if last.get(site, -1) > g:
                raise ValueError(f"layer {layer}: mode {mode} follows a later layer's beam splitter on site {site}")
            last[site] = g
        groups[layer].append((int(mode), float(th), float(ph)))
    out = []
    for layer in order:
        g = groups[layer]
        out.append(([x[0] for x in g], [x[1] for x in g], [x[2] for x in g]))
    return out


def block_owner(n, layers, world):
    """Rank of every mode 0..n-2: contiguous blocks in mode order, balanced by the number
    of beam splitters on each mode (a mode with no beam splitter counts one half)."""
    count = np.zeros(n - 1)
    for modes, _, _ in layers:
        for m in modes:
            count[m] += 1.0
    w = np.maximum(count, 0.5)
    mid = np.cumsum(w) - 0.5 * w
    owner = np.minimum((mid * world / w.sum()).astype(np.int64), world - 1)
    return [int(r) for r in owner]


class HaloPlan:
    """Exchange schedule of a brick-wall mesh over ``world`` ranks.

    ``owner[m]`` runs the beam splitter on (m, m+1).  ``transfers[l]`` lists, for layer
    l, the ``((kind, index), src, dst)`` copies that must land before the layer's updates
    run; ``gather`` lists the copies that bring every current site and bond to ``root``
    after the last layer.  Each item's source is the rank that last wrote it, or, for an
    item no update wrote yet, the lowest-ranked holder of the replicated initial state.
    """

    def __init__(self, n, layers, world, owner=None, root=0):
        if world < 1:
            raise ValueError("world must be >= 1")
        self.n, self.world, self.root = int(n), int(world), int(root)
        self.layers = [(list(m), list(t), list(p)) for m, t, p in layers]
        for l, (modes, _, _) in enumerate(self.layers):
            sites = set()
            for m in modes:
                if not 0 <= m <= self.n - 2:
                    raise ValueError(f"layer {l}: mode {m} out of range")
                if m in sites or m + 1 in sites:
                    raise ValueError(f"layer {l}: beam splitters on overlapping sites (not a brick-wall layer)")
                sites.update((m, m + 1))
        self.owner = list(owner) if owner is not None else block_owner(self.n, self.layers, self.world)
        if len(self.owner) != self.n - 1 or any(not 0 <= r < self.world for r in self.owner):
            raise ValueError("owner must give a rank in [0, world) for each of the n-1 modes")
        items = [(SITE, i) for i in range(self.n)] + [(BOND, b) for b in range(1, self.n)]
        fresh = {it: set(range(self.world)) for it in items}   # ranks holding the current version
        writer = {}
        self.transfers = []
        for l, (modes, _, _) in enumerate(self.layers):
            tr = []
            for m in modes:
                r = self.owner[m]
                for it in _reads(self.n, m):
                    if r not in fresh[it]:
                        src = writer.get(it, min(fresh[it]))
                        tr.append((it, src, r))
                        fresh[it].add(r)
            for m in modes:
                r = self.owner[m]
                for it in _writes(m):
                    fresh[it] = {r}
                    writer[it] = r
            self.transfers.append(tr)
        self.gather = [(it, writer.get(it, min(fresh[it])), self.root) for it in items if self.root not in fresh[it]]

    def local_layer(self, l, rank):
        """(modes, thetas, phis) of layer l that ``rank`` runs, in mesh order."""
        modes, th, ph = self.layers[l]
        keep = [i for i, m in enumerate(modes) if self.owner[m] == rank]
        return [modes[i] for i in keep], [th[i] for i in keep], [ph[i] for i in keep]

    def bytes_moved(self, chi):
        """Bytes the layers' exchanges and the final gather move (Gamma chi^2 x 16,
        a bond chi x (8 + 8))."""
        size = {SITE: chi * chi * 16, BOND: chi * 16}
        per_layer = [sum(size[it[0]] for it, _, _ in tr) for tr in self.transfers]
        return per_layer, sum(size[it[0]] for it, _, _ in self.gather)


class DeviceSites:
    """A rank's state: one ``MPOSimulator`` handle holding the whole chain's layout, on
    the CUDA device that was current when it was made (every call runs there)."""

    def __init__(self, sim):
        self.sim = sim
        self.device = sim.torch.cuda.current_device()

    def export(self, item):
        kind, idx = item
        with self.sim.torch.cuda.device(self.device):
            if kind == SITE:
                return [self.sim.get_site(idx)]
            return list(self.sim.get_bond(idx))

    def buffers(self, item):
        t = self.sim.torch
        dev = t.device("cuda", self.device)
        chi = self.sim.chi
        if item[0] == SITE:
            return [t.empty((chi, chi), dtype=t.complex128, device=dev)]
        return [t.empty(chi, dtype=t.float64, device=dev), t.empty((chi, 2), dtype=t.int32, device=dev)]

    def receive(self, item, tensors):
        kind, idx = item
        with self.sim.torch.cuda.device(self.device):
            if kind == SITE:
                self.sim.put_site(idx, tensors[0])
            else:
                self.sim.put_bond(idx, tensors[0], tensors[1])

    def run(self, modes, thetas, phis):
        if modes:
            with self.sim.torch.cuda.device(self.device):
                self.sim.run_mesh(modes, thetas, phis)

    def synchronize(self):
        self.sim.torch.cuda.synchronize(self.device)


class DistTransport:
    """``torch.distributed`` point-to-point between this rank and its neighbours (NCCL
    between GPUs, gloo between host processes): one message per array, all of a layer's
    messages posted together (``batch_isend_irecv``) and waited for before the received
    items are copied in."""

    def __init__(self, rank=None):
        import torch.distributed as dist
        self.dist = dist
        self.rank = dist.get_rank() if rank is None else int(rank)

    def exchange(self, transfers, sites):
        dist, me = self.dist, self.rank
        mine = sites[me]
        ops, landing = [], []
        for it, src, dst in transfers:
            if src == dst:
                continue
            if src == me:
                for x in mine.export(it):
                    ops.append(dist.P2POp(dist.isend, x, dst))
            elif dst == me:
                bufs = mine.buffers(it)
                landing.append((it, bufs))
                for x in bufs:
                    ops.append(dist.P2POp(dist.irecv, x, src))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        mine.synchronize()
        for it, bufs in landing:
            mine.receive(it, bufs)


class LocalTransport:
    """Several ranks' states driven by one process: each transfer is a direct copy from
    the source rank's state into the destination's (a peer copy when they sit on
    different GPUs)."""

    def exchange(self, transfers, sites):
        for it, src, dst in transfers:
            if src == dst:
                continue
            bufs = sites[dst].buffers(it)
            for b, x in zip(bufs, sites[src].export(it)):
                b.copy_(x)
            sites[dst].synchronize()
            sites[dst].receive(it, bufs)


class HaloCircuit:
    """Runs the layers of a ``HaloPlan`` on the ranks' states ``sites`` ({rank: state};
    under ``DistTransport`` only this rank's), exchanging before each layer and gathering
    every current site and bond on the plan's root at the end."""

    def __init__(self, plan, sites, transport):
        self.plan, self.sites, self.transport = plan, dict(sites), transport

    def run(self):
        for l in range(len(self.plan.layers)):
            self.transport.exchange(self.plan.transfers[l], self.sites)
            for r, st in self.sites.items():
                st.run(*self.plan.local_layer(l, r))
        self.transport.exchange(self.plan.gather, self.sites)
        for st in self.sites.values():
            st.synchronize()


def run_distributed(n, d, chi, photon_modes, eta, mesh, phases, precision="fp64-gram", workers=16):
    """The whole circuit on the ranks of the initialised default process group (one
    process per GPU, ``torch.cuda.set_device`` done): every rank builds the same initial
    state, runs its block of each layer with the halo exchange, and the root gathers
    the state, applies the output phases and computes the observables.  Returns
    ``(trace, marginals)`` on the root and None elsewhere."""
    import torch.distributed as dist

    from .engine import MPOSimulator
    rank, world = dist.get_rank(), dist.get_world_size()
    plan = HaloPlan(n, layers_of(mesh), world)
    with MPOSimulator(n, d, chi) as sim:
        sim.set_precision(precision)
        sim.set_workers(workers)
        sim.init_single_photons(photon_modes, eta)
        dist.barrier()   # every rank joins the communicator before the first exchange
        HaloCircuit(plan, {rank: DeviceSites(sim)}, DistTransport(rank)).run()
        if rank != plan.root:
            return None
        sim.apply_phases(phases)
        return sim.observables()
