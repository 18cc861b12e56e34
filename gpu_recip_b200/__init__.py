"""gpu_recip_b200 -- B200-native smooth-PME reciprocal-space engine.

The compute path is the CUDA library libpme_b200.so (sm_100a kernels behind the C ABI of
include/pme_recip.h); this package is its Python front end, mirroring the reference operator
interface (CudaPMERecip / CudaDomdecRecip of ap-hynninen/gpu_recip).
"""
from . import _capi
from .pme import (CCELEC, FFT_BOX, FFT_COLUMN, FFT_SLAB, FORCE_SCALE, CudaDomdecRecip,
                  CudaPMERecip, EnergyVirial, PmeBatch, PmeServer, force_convert, force_convert_add,
                  force_stride, recip_from_box, recip_from_box_vectors, system_device_bytes)

__all__ = ["CudaPMERecip", "CudaDomdecRecip", "EnergyVirial", "PmeBatch", "PmeServer", "recip_from_box",
           "recip_from_box_vectors", "force_stride", "force_convert", "force_convert_add", "system_device_bytes",
           "FFT_BOX", "FFT_COLUMN", "FFT_SLAB", "CCELEC", "FORCE_SCALE", "load_library"]


def load_library():
    """Load the CUDA library; raises if it was not built (there is no CPU fallback)."""
    return _capi.load()
