"""B200-native beam-splitter update of a U(1)-symmetric density-matrix MPO.

The hot path (Fock beam-splitter tensor -> charge-block contraction -> per-sector
SVD -> top-chi truncation) runs as sm_100a CUDA kernels in ``libbsmpo.so``
(C ABI: ``include/bsmpo.h``).  Python modules mirror the reference simulator's call
surface:

* ``cuda_kernels``  -- ``Rand_U``, ``update_MPO`` (reference ``src/cuda_kernels.py``)
* ``MPO``           -- ``Initialize`` (reference ``src/MPO.py:21-134``)
* ``summary``       -- ``Probability``, ``EntanglementEntropy`` (``src/summary.py``)
* ``gpu_algorithm`` -- ``Worker`` with the ``run.py`` protocol
* ``engine``        -- ``MPOSimulator``, the device-resident simulator
"""
from .engine import MPOSimulator  # noqa: F401
