"""CPU oracle for the beam-splitter MPO update (TEST INFRASTRUCTURE ONLY).

This package is a plain numpy (complex128 / float64) restatement of the reference
simulator's CPU algorithm for the beam-splitter update of a U(1)-symmetric
density-matrix MPO:

* ``fock``           -- two-mode Fock beam-splitter tensor
                        (reference ``src/MPO.py:6-18``, ``src/u_kernel.cu:37-71``)
* ``interferometer`` -- seeded Haar unitary and its Clements rectangular mesh
* ``mpo``            -- initial product MPO + canonicalising sweep
                        (``src/MPO.py:21-155``), the two-site charge-block update
                        (``src/MPO.py:158-303``) and the observables
                        (``src/summary.py:3-36``)
* ``circuit``        -- runs a whole mesh BS by BS (``src/beam_splitter_parallel/Full.py:149-202``)

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import it, and only as the checker / the timed CPU baseline.  The product
path (``bosonsampling_b200``) never imports it.

Parity pin: the restatement is checked against the reference's own ``src/MPO.py``
(imported in the build container with a stub ``qutip``) through the committed
fixtures in ``tests/golden/`` and the script that generated them
(``tests/golden/make_golden.py``).
"""
