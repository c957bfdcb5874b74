"""CPU oracle for the SLEvolve per-time-step sea-level path.

TEST INFRASTRUCTURE ONLY.  This package is a NumPy restatement of the reference
algorithm (SLEvolve ``python/slevolve/sht.py``, ``solver.py`` and the parts of
``solver_opt.py`` that the GPU path implements).  It exists to check the CUDA
implementation in ``slevolve_b200``; it is never the thing measured or shipped.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  The product path (``slevolve_b200``) never imports
anything from here and fails loudly when its CUDA library is missing.

Parity pin: ``tests/golden/make_golden.py`` runs the reference Python solver
(imported from a checkout of the reference) on seeded inputs and commits the
outputs as fixtures under ``tests/golden/``; ``tests/test_oracle_golden.py``
checks this oracle against those fixtures, and ``tests/golden/synthetic512``
records the oracle against the reference's own shipped golden grid
(``reference/synthetic/tgrid8.npy``).

Modules
-------
``oracle.sht``     Gauss-Legendre nodes, normalised Legendre functions and the
                   spectral transform (sht.py:65-343).
``oracle.memory``  the recursive modal state (solver.py:244-506).
``oracle.solver``  the time step (solver.py:521-1144; solver_opt.py:148-165 for
                   the extrapolated inner start, 320-325 for the ``dsl``
                   identity, the ``diag`` degree-0 row-sum quadrature).
"""
