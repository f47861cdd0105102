"""``gpu_algorithm.Worker``: the single-GPU worker ``run.py`` expects.

The reference's ``src/gpu_algorithm/__init__.py`` is empty although ``run.py:37-43``
calls ``gpu_algorithm.Worker()``; this fills that protocol with the device-resident
simulator.  The brick-wall walk is the one of ``src/beam_splitter_parallel/Full.py``
(``LayerUpdate`` :149-166, ``Simulate`` :169-202): layer l applies the beam splitters
on (m, m+1), m = l mod 2, then records the trace and the per-bond entanglement
entropy.  The mesh is the Clements decomposition of a seeded Haar unitary (the
reference's own mesh generator, ``src/interferometer.py``, draws reflectivities from
a custom pdf instead), and every mesh beam splitter is applied (no light-cone skip).
"""
import numpy as np

from . import interferometer
from .engine import MPOSimulator, lossy_single_photon_rhos
from .summary import EntanglementEntropy


class Worker:
    def __init__(self):
        self.sim = None

    def ExperimentInit(self, input_state_type, n_modes, n_input_states, post_selected_photon_number,
                       local_hilbert_space_dimension, bond_dimension, parameters, seed=None,
                       photon_modes=None):
        if input_state_type != "Single photon":
            raise NotImplementedError("input_state_type %r is outside the single-photon workloads" % input_state_type)
        self.n_modes = int(n_modes)
        self.d = int(local_hilbert_space_dimension)
        self.chi = int(bond_dimension)
        self.prob = np.zeros([self.n_modes + 1], dtype="float32")
        self.EE = np.zeros([self.n_modes - 1, self.n_modes + 1], dtype="float32")
        self.REPar = np.zeros([self.n_modes - 1, self.n_modes + 1, 5], dtype="float32")
        self.U, bs, self.out_phases = interferometer.circuit(self.n_modes, 0 if seed is None else int(seed))
        self.layers = [[] for _ in range(self.n_modes)]
        for (layer, m, th, ph) in bs:
            self.layers[layer].append((m, th, ph))
        modes = list(range(n_input_states)) if photon_modes is None else list(photon_modes)
        eta = 1.0 - float(parameters["loss"])
        if self.sim is not None:
            self.sim.close()
        self.sim = MPOSimulator(self.n_modes, self.d, self.chi)
        self.sim.init_product(lossy_single_photon_rhos(self.n_modes, modes, eta, self.d),
                              total_photons=post_selected_photon_number)
        self.prob[0] = self.sim.trace().real
        self.initialization_successful = bool(self.prob[0] > 0)

    def _lambdas(self):
        _, lam, _ = self.sim.store()
        return lam

    def Simulate(self):
        success = True
        if self.initialization_successful:
            self.EE[:, 0] = EntanglementEntropy(self._lambdas())
            for layer in range(self.n_modes):
                ops = self.layers[layer]
                if ops:
                    self.sim.run_mesh([m for (m, _, _) in ops], [t for (_, t, _) in ops],
                                      [p for (_, _, p) in ops])
                self.prob[layer + 1] = self.sim.trace().real
                self.EE[:, layer + 1] = EntanglementEntropy(self._lambdas())
        return success, self.prob, self.EE, self.REPar
