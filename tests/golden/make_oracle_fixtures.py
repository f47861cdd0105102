"""Generate oracle fixtures for the full seeded workloads (CPU, no GPU needed).

    python tests/golden/make_oracle_fixtures.py [plain-small] [plain-scale] [precision-l11]

Runs the CPU oracle (oracle/) over the whole Clements mesh of each workload and
stores the final trace, single-mode marginals, per-bond Lambda spectra (with their
charges) and the per-update truncation weights, so GPU parity tests at these sizes
do not have to rerun the oracle (the 496-update workload takes minutes on a CPU).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import circuit, interferometer, mpo  # noqa: E402


# Bounded runs of the large workload: the first `layers` brick-wall layers only (the
# bond dimension saturates at chi = 1024 from layer 5 on).  Phases and the rest of the
# mesh are not applied; trace and marginals do not depend on output phases anyway.
PARTIAL = {"precision-l11": ("precision", 11)}


def main(names):
    for name in names:
        base, n_layers = PARTIAL.get(name, (name, None))
        w = circuit.WORKLOADS[base]
        t0 = time.time()
        infos = []
        max_bs = None
        if n_layers is not None:
            _, bs_all, _ = interferometer.circuit(w["n"], w["seed"])
            max_bs = sum(1 for b in bs_all if b[0] < n_layers)
        st, U, bs = circuit.run(**w, infos=infos, max_bs=max_bs)
        P = mpo.marginals(st)
        out = dict(
            n=w["n"], eta=w["eta"], d=w["d"], chi=w["chi"], seed=w["seed"],
            trace=np.array([mpo.trace(st)]), marginals=P,
            lam=st.Lambda, charge=st.charge,
            trunc_weight=np.array([i.trunc_weight for i in infos]),
            # total sigma^2 of each update: the scale of its truncation-weight tolerance
            total_weight=np.array([sum(float(np.sum(s ** 2)) for s in i.sigma) for i in infos]),
            bond_dims=np.array(mpo.bond_dims(st)),
            n_bs=np.array([len(infos)]),
        )
        path = os.path.join(HERE, "oracle_%s.npz" % name.replace("-", "_"))
        np.savez_compressed(path, **out)
        print(name, "%.1f s" % (time.time() - t0), "trace", out["trace"][0], "->", path,
              os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1:] or ["plain-small", "plain-scale"])
