"""Golden fixture of the reference's own update at the benchmarked size.

Run in the build container (it reads the reference checkout; nothing at test time does):

    python tests/golden/make_ref_chi1024.py /path/to/reference

Workload: N = 64 modes, lossy single photons (eta = 0.3) in the even modes, d = 5,
chi = 1024, the Clements mesh of Haar seed 1003.  The oracle advances it through layers
0-5 (every bond holds 1024 values from layer 5 on) and through layer 6's updates left of
mode 24.  The next four updates of layer 6 then run in the reference's
``InitializationMPO.Update`` (``src/MPO.py:158-303``, complex64, loaded in memory as
``make_golden.py`` loads it), each from the oracle's state at that point.  The
reference's new centre bond (Lambda and charges) is recorded for each update, with a
flag where the reference's cut split a ket/bra-swapped sector pair.
``tests/test_oracle_golden.py`` checks that the oracle's update reproduces it.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from oracle import fock, interferometer, mpo  # noqa: E402
from oracle.time_reference_cpu import refresh, to_reference  # noqa: E402

N, D, CHI, ETA, SEED, LAYER, FIRST_MODE, UPDATES = 64, 5, 1024, 0.3, 1003, 6, 24, 4


def oracle_start():
    """The oracle's state just before the recorded updates, and those updates."""
    _, bs, _ = interferometer.circuit(N, SEED)
    st = mpo.initial_state(N, range(0, N, 2), ETA, D, CHI)
    for layer, m, th, ph in bs:
        if layer < LAYER or (layer == LAYER and m < FIRST_MODE):
            mpo.bs_update(st, m, fock.update_tensor(interferometer.t_block(th, ph), D))
    timed = [(m, th, ph) for layer, m, th, ph in bs if layer == LAYER and m >= FIRST_MODE][:UPDATES]
    return st, timed


def main(ref_root):
    from make_golden import load_reference, swap_symmetric
    ref, _ = load_reference(ref_root)
    st, timed = oracle_start()
    obj = object.__new__(ref.InitializationMPO)
    obj.n_modes, obj.local_hilbert_space_dimension, obj.bond_dimension = N, D, CHI
    obj.edge_Lambda = np.ones(CHI, dtype="float32")
    to_reference(st, obj)
    modes, lams, chgs, splits = [], [], [], []
    for m, th, ph in timed:
        U3 = fock.update_tensor(interferometer.t_block(th, ph), D)
        obj.Unitary = fock.tensor3_to_4(U3).astype(np.complex64)
        obj.Update(m)
        # the reference keeps an arbitrary member of a ket/bra-swapped pair that the cut
        # splits (the oracle keeps neither): recorded, the test compares around it
        splits.append(not swap_symmetric(obj.charge[:, m + 1, :], obj.Lambda[:, m], D))
        modes.append(m)
        lams.append(obj.Lambda[:, m].astype(np.float64))
        chgs.append(obj.charge[:, m + 1, :].astype(np.int32))
        mpo.bs_update(st, m, U3)
        refresh(st, obj, m)
    path = os.path.join(HERE, "ref_chi1024_layer6.npz")
    np.savez_compressed(path, n=N, d=D, chi=CHI, eta=ETA, seed=SEED, layer=LAYER, first_mode=FIRST_MODE,
                        mode=np.array(modes, dtype=np.int32), ref_lambda=np.array(lams),
                        ref_charge=np.array(chgs), ref_split_pair=np.array(splits))
    print(path, modes, "split pairs", splits, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_ref_chi1024.py <path of the reference checkout>")
    main(sys.argv[1])
