"""Whole-circuit driver for the CPU oracle (test infrastructure only).

Walks the Clements mesh BS by BS in brick-wall layer order -- the reference's
``LayerUpdate``/``Simulate`` walk (``src/beam_splitter_parallel/Full.py:149-202``),
without its light-cone skip (``:153``), which is only valid for inputs packed into the
first modes -- and finishes with the output phase screen and the observables.
"""
import time

import numpy as np

from . import fock, interferometer, mpo

# Synthetic workloads: (modes, transmissivity, cutoff d, bond dim chi, Haar seed).
WORKLOADS = {
    "plain-small": dict(n=16, eta=0.5, d=4, chi=64, seed=1001),
    "plain-scale": dict(n=32, eta=0.5, d=4, chi=256, seed=1002),
    "precision": dict(n=64, eta=0.3, d=5, chi=1024, seed=1003),
    "diff": dict(n=24, eta=0.5, d=4, chi=256, seed=1005),
}


def even_modes(n):
    return list(range(0, n, 2))


def gate_tensors(bs_list, d):
    """U[new_a, new_b, old_a] for every mesh BS (T(theta, phi) acting on the state)."""
    return [fock.update_tensor(interferometer.t_block(th, ph), d) for (_, _, th, ph) in bs_list]


def run(n, eta, d, chi, seed, photon_modes=None, max_bs=None, infos=None, phases=True, cutoff=0.0):
    """Run the mesh of the seeded Haar unitary; returns (state, U, bs_list)."""
    U, bs, ph = interferometer.circuit(n, seed)
    if photon_modes is None:
        photon_modes = even_modes(n)
    st = mpo.initial_state(n, photon_modes, eta, d, chi)
    todo = bs if max_bs is None else bs[:max_bs]
    for (layer, m, th, phi) in todo:
        U3 = fock.update_tensor(interferometer.t_block(th, phi), d)
        info = mpo.bs_update(st, m, U3, cutoff=cutoff)
        if infos is not None:
            infos.append(info)
    if phases and max_bs is None:
        mpo.apply_phases(st, ph)
    return st, U, bs


def timed_sample(n, eta, d, chi, seed, budget_s=15.0, photon_modes=None):
    """Run BS updates until ``budget_s`` of CPU time is spent; returns (n_bs, seconds)."""
    U, bs, ph = interferometer.circuit(n, seed)
    if photon_modes is None:
        photon_modes = even_modes(n)
    st = mpo.initial_state(n, photon_modes, eta, d, chi)
    t0 = time.perf_counter()
    done = 0
    for (layer, m, th, phi) in bs:
        U3 = fock.update_tensor(interferometer.t_block(th, phi), d)
        mpo.bs_update(st, m, U3)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    return done, time.perf_counter() - t0
