"""Host side of the B200 FDTD S-parameter engine (``liboidt.so``, sm_100a).

* ``engine`` -- ctypes binding of the C ABI (``include/oidt.h``): ``Engine``
  (one context per device) and ``Job`` (one simulation's device state).
* ``spec`` -- the job description (``SimSpec``) and its ABI descriptor.
* ``refsetup`` -- the reference's setup from its user dictionaries;
  ``workloads`` -- synthetic guides with explicit sizes.
* ``fdtd_main``, ``extract_sparams``, ``simulation_launcher`` -- drop-ins for
  the reference's three S-parameter scripts; ``sparams`` -- S-matrices and
  touchstone files.
* ``batch`` -- batched roughness realizations; ``serve`` -- the continuous-
  batching request loop; ``tune`` -- per-shape launch choices.
* ``scatter``, ``zwave`` -- the scattering-loss and wave-impedance
  workloads; ``large`` -- the 151 M-cell run (profiler cases are
  ``bench.py --ncu-case``).
* ``build`` -- compiles ``liboidt.so`` in-tree.

Nothing here falls back to the CPU: without the library, ``engine`` raises.
"""
