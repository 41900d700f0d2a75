"""CPU oracle for the OIDT FDTD S-parameter path -- TEST INFRASTRUCTURE ONLY.

This package restates, in float64 NumPy (``fdtd_ref``) and in plain C
(``c/oracle.c``), the reference's GPU S-parameter extraction loop:

* setup      ``FDTD/GPU/FDTD_2D_TM/s-parameter_extraction/fdtd_auto_setup.py:42-170``
             ``FDTD/GPU/FDTD_3D/s-parameter_extraction/fdtd_auto_setup.py:42-177``
* geometry + coefficients + CPML grading
             ``FDTD/GPU/FDTD_2D_TM/s-parameter_extraction/fdtd_main.py:51-178``
             ``FDTD/GPU/FDTD_2D_TE/s-parameter_extraction/fdtd_main.py:51-180``
             ``FDTD/GPU/FDTD_3D/s-parameter_extraction/fdtd_main.py:51-221``
* kernels    ``FDTD/GPU/FDTD_2D_TM/s-parameter_extraction/fdtd_funcs.py:43-144``
             ``FDTD/GPU/FDTD_2D_TE/s-parameter_extraction/fdtd_funcs.py:43-152``
             ``FDTD/GPU/FDTD_3D/s-parameter_extraction/fdtd_funcs.py:43-302``
* time loop  ``FDTD/GPU/FDTD_2D_TM/s-parameter_extraction/fdtd_main.py:275-304``
             ``FDTD/GPU/FDTD_3D/s-parameter_extraction/fdtd_main.py:357-406``
* extraction ``FDTD/GPU/FDTD_2D_TM/s-parameter_extraction/extract_sparams.py:48-117``
             ``FDTD/GPU/FDTD_3D/s-parameter_extraction/extract_sparams.py:48-144``

Parity is pinned: ``tests/golden/make_golden.py`` runs the reference's own
``fdtd_main.py`` under Numba's CUDA simulator in float64 and records its
device arrays; ``tests/test_oracle_golden.py`` requires this oracle to
reproduce them bit for bit.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import, call, link or execute anything in this package, and only as
the reference results the tests compare against or the timed CPU baseline.  The product (``oidt_b200``) never
imports it and has no CPU fallback.
"""
