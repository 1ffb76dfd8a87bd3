"""viprs_b200: B200-native (sm_100a) resample path of viprs.

The product is the in-tree shared library viprs_b200/_lib/libviprs_b200.so
(C ABI declared in include/viprs_b200.h).  This package is its Python face:
``viprs_b200.api`` mirrors viprs's PipelineBuilder ops over torch CUDA
tensors.  Importing the package does not load the library; the first call
does, and fails loudly if it was not built.
"""
from . import _native  # noqa: F401

__version__ = "0.1.0"
