"""srsoriginal_b200: B200-native radiation hot path of the SRS / OSCARS simulator.

``srsoriginal_b200.sr.sr`` is the reference's ``oscars.sr.sr`` type for the hot-path calls; the
C ABI of ``libsrs_b200.so`` (include/srs_b200.h) is the drop-in boundary underneath it.
"""
__version__ = "1.0.0"
