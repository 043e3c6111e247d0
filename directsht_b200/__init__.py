"""B200-native DirectSHT forward transform (drop-in for martinjameswhite/directsht).

``DirectSHT`` mirrors the reference's ``sht.sht.DirectSHT``; the arithmetic runs in the
sm_100a kernels of ``libdsht_b200.so`` (C ABI in ``include/dsht.h``).
"""
from .sht import DirectSHT  # noqa: F401

__all__ = ["DirectSHT"]
__version__ = "0.1.0"
