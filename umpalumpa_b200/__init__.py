"""B200-native Fourier reconstruction (Umpalumpa AFR drop-in).

The product is the CUDA engine behind the C-ABI in include/umpalumpa_fr.h and
include/umpalumpa_fr_server.h, built into umpalumpa_b200/lib/libfr_b200.so.

* ``umpalumpa_b200.fr`` -- the reference operation API for Python callers (FRB200: Init /
  Execute / Synchronize), the batched form (FRBatch), the autotuner, input preparation (Prep),
  traverse spaces with and without symmetry operations, 16-bit quantisation;
* ``umpalumpa_b200.server`` -- the serving form (FRServer) and one server per GPU (ServerPool);
* ``umpalumpa_b200.parallel`` -- projection sharding and the sum reduction across ranks;
* ``umpalumpa_b200.synthetic`` -- seeded test and bench jobs and the served-workload trace.
"""
__version__ = "0.1.0"
