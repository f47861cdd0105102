"""Drop-in for the reference's ``src/MPO.py`` state construction.

``Initialize`` builds the product MPO on the host (tiny: bond dimension <= d) and
canonicalises it on the device with the same update kernels the simulation uses.
"""
import numpy as np

from .engine import MPOSimulator, lossy_single_photon_rhos


def Initialize(input_state_type, n_modes, n_input_states, post_selected_photon_number,
               local_hilbert_space_dimension, parameters, bond_dimension=None,
               photon_modes=None):
    """Initial MPO as ``Initialize`` (``src/MPO.py:21-134``).

    'Single photon' inputs: vacuum weight ``parameters['loss']`` (the reference's
    convention; transmissivity eta = 1 - loss) on the first ``n_input_states`` modes,
    or on ``photon_modes`` when given.  Returns host arrays ``Gamma[n, chi, chi]``
    complex128, ``Lambda[n-1, chi]`` float64 and ``charge[n+1, chi, 2]`` int32
    (sentinel d on empty slots), chi = ``bond_dimension`` or d^2 (the reference's).
    """
    d = int(local_hilbert_space_dimension)
    if input_state_type == "Single photon":
        loss = parameters["loss"]
    elif input_state_type in ("Gaussian", "Thermal"):
        raise NotImplementedError("input_state_type %r is outside the single-photon workloads" % input_state_type)
    else:
        raise ValueError("input_state_type {} not supported.".format(input_state_type))
    chi = int(bond_dimension) if bond_dimension is not None else d * d
    modes = list(range(n_input_states)) if photon_modes is None else list(photon_modes)
    with MPOSimulator(n_modes, d, chi) as sim:
        sim.init_product(lossy_single_photon_rhos(n_modes, modes, 1.0 - loss, d),
                         total_photons=post_selected_photon_number)
        g, l, c = sim.store()
        return g.cpu().numpy(), l.cpu().numpy(), c.cpu().numpy()
