"""B200-native DirectSHT forward transform (drop-in for martinjameswhite/directsht).

``DirectSHT`` mirrors the reference's ``sht.sht.DirectSHT`` and ``MaskDeconvolution`` its
``sht.mask_deconvolution.MaskDeconvolution``; the arithmetic runs in the sm_100a kernels of
``libdsht_b200.so`` (C ABI in ``include/dsht.h``).
"""
from .mask import MaskDeconvolution  # noqa: F401
from .sht import DirectSHT  # noqa: F401

__all__ = ["DirectSHT", "MaskDeconvolution"]
__version__ = "0.1.0"
