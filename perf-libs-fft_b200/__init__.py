"""plfft_b200: B200-native batched 1D FFT behind the plfft.h C-ABI.

The product is ``lib/libplfft_b200.so`` (CUDA kernels + C-ABI, built from
``csrc/`` by the Makefile).  ``plfft.py`` is the Python mirror of the C API.
"""
from .plfft import *  # noqa: F401,F403
