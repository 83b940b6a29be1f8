"""CPU oracle for the forward-model hot path (TEST INFRASTRUCTURE ONLY).

This package restates, in NumPy, the reference's USFFT Radon pair
(``processing/tomo.py`` / ``processing/tomo_large.py``), its Fresnel
propagator (``processing/propagation.py`` / ``processing/propagation_large.py``)
and the two elementwise stages of ``step3_propagation.py``.  It exists to
check the CUDA product path and is used only by ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py``.  The product (``model_mosaic_b200``) never imports it.

Parity pin: ``oracle/build_ref.py`` compiles the reference's own kernel source
(``processing/kernels.py``) for the host; ``tests/golden/make_golden.py`` runs
those kernels with this package's FFT glue to produce the committed fixtures
under ``tests/golden/``, and ``tests/test_oracle.py`` checks this restatement
against them.
"""
