"""B200-native Fourier reconstruction (Umpalumpa AFR drop-in).

The product is the CUDA engine behind the C-ABI in include/umpalumpa_fr.h, built into
umpalumpa_b200/lib/libfr_b200.so.  ``umpalumpa_b200.fr`` mirrors the reference operation API
for Python callers; ``umpalumpa_b200.synthetic`` makes seeded test/bench jobs.
"""
__version__ = "0.1.0"
