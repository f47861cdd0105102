"""Times the reference's own CPU update beside the oracle port, on the same state of the
benchmark workload (test infrastructure; run where the reference checkout exists):

    python oracle/time_reference_cpu.py /path/to/reference [--start-layer 10] [--updates 6] [--first-mode 24]

The reference's update is ``InitializationMPO.Update`` (``src/MPO.py:158-303``: numpy,
complex64 state, float32 Lambda), loaded in memory as the golden-fixture generator loads
it.  The port is ``oracle.mpo.bs_update`` (FP64).  The workload is N = 64 modes, lossy
single photons (eta = 0.3) in the even modes, d = 5, chi = 1024, the Clements mesh of Haar
seed 1003, advanced by the port to ``--start-layer``.  Each timed update starts both
implementations from the port's current state (the reference's arrays are refreshed
from it on the sites and bonds the previous update changed), so the two are timed on
identical inputs; the largest relative difference of the new centre-bond Lambda
between them is printed with each time.  Both run on all host cores (numpy's BLAS
threads).
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "tests", "golden"))

from oracle import fock, interferometer, mpo  # noqa: E402


def to_reference(st, obj):
    """Copy the port's state into the reference's internal layout
    (Gamma [chi, chi, n] complex64, Lambda [chi, n-1] float32, charge [chi, n+1, 2])."""
    obj.Gamma = np.ascontiguousarray(np.transpose(st.Gamma, (1, 2, 0))).astype(np.complex64)
    obj.Lambda = np.ascontiguousarray(st.Lambda.T).astype(np.float32)
    obj.charge = np.ascontiguousarray(np.transpose(st.charge, (1, 0, 2))).astype(np.int32)


def refresh(st, obj, mode):
    """Bring the sites and bond an update on ``mode`` changed back to the port's values."""
    for s in (mode, mode + 1):
        obj.Gamma[:, :, s] = st.Gamma[s].astype(np.complex64)
    obj.Lambda[:, mode] = st.Lambda[mode].astype(np.float32)
    obj.charge[:, mode + 1, :] = st.charge[mode + 1]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("reference")
    ap.add_argument("--start-layer", type=int, default=10)
    ap.add_argument("--updates", type=int, default=6)
    ap.add_argument("--first-mode", type=int, default=24,
                    help="time the layer's updates from this mode on (the centre, where the bonds are full)")
    a = ap.parse_args()
    from make_golden import load_reference
    ref, _ = load_reference(a.reference)

    n, d, chi, eta, seed = 64, 5, 1024, 0.3, 1003
    _, bs, _ = interferometer.circuit(n, seed)
    t0 = time.perf_counter()
    st = mpo.initial_state(n, range(0, n, 2), eta, d, chi)
    ops = [(m, th, ph) for (layer, m, th, ph) in bs if layer < a.start_layer]
    for m, th, ph in ops:
        mpo.bs_update(st, m, fock.update_tensor(interferometer.t_block(th, ph), d))
    print("advanced %d updates to layer %d in %.0f s" % (len(ops), a.start_layer, time.perf_counter() - t0), flush=True)

    obj = object.__new__(ref.InitializationMPO)
    obj.n_modes, obj.local_hilbert_space_dimension, obj.bond_dimension = n, d, chi
    obj.edge_Lambda = np.ones(chi, dtype="float32")
    to_reference(st, obj)
    later = [(layer, m, th, ph) for (layer, m, th, ph) in bs if layer >= a.start_layer]
    # the start layer's updates left of --first-mode run untimed (on the port; the
    # reference's arrays follow it), the next --updates ones are timed
    first = next(i for i, (layer, m, _, _) in enumerate(later) if layer > a.start_layer or m >= a.first_mode)
    for _, m, th, ph in later[:first]:
        mpo.bs_update(st, m, fock.update_tensor(interferometer.t_block(th, ph), d))
        refresh(st, obj, m)
    timed = [(m, th, ph) for (_, m, th, ph) in later[first:first + a.updates]]
    t_ref, t_port = [], []
    for m, th, ph in timed:
        U3 = fock.update_tensor(interferometer.t_block(th, ph), d)
        obj.Unitary = fock.tensor3_to_4(U3).astype(np.complex64)
        t = time.perf_counter()
        obj.Update(m)
        t_ref.append(time.perf_counter() - t)
        lam_ref = obj.Lambda[:, m].astype(np.float64)
        t = time.perf_counter()
        mpo.bs_update(st, m, U3)
        t_port.append(time.perf_counter() - t)
        lam = st.Lambda[m]
        k = min(np.count_nonzero(lam), np.count_nonzero(lam_ref))
        diff = np.abs(np.sort(lam_ref)[::-1][:k] - np.sort(lam)[::-1][:k]).max() / lam.max()
        print("mode %2d  reference %.2f s  port %.2f s  centre-bond Lambda rel. diff %.1e"
              % (m, t_ref[-1], t_port[-1], diff), flush=True)
        refresh(st, obj, m)
    cores = len(os.sched_getaffinity(0))
    print("reference (complex64): %.3f BS-updates/s; port (FP64): %.3f BS-updates/s; %d cores; %d updates"
          % (len(t_ref) / sum(t_ref), len(t_port) / sum(t_port), cores, len(t_ref)))


if __name__ == "__main__":
    main()
