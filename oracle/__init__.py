"""CPU oracle for the SmallStrainFFT path (test infrastructure only).

This package is the checker, never the product: only ``tests/``, the smoke check in
``__graft_entry__`` and the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``
may import it.  It restates, in numpy, the algorithm of materialite 0.1.3's
``SmallStrainFFT`` solve (``materialite/models/small_strain_fft/*.py``) on plain arrays.

Parity pins: ``tests/test_oracle.py`` checks it against the reference's own known-answer
tests (``tests/test_elastic_model.py``, ``tests/test_elastic_viscoplastic_model.py``,
``tests/test_hardening_laws.py``) and against golden fields produced by running the
reference itself (``tests/golden/make_golden.py``).
"""
