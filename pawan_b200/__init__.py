"""B200-native vortex-particle hot path of PAWAN (PArticle Wake ANalysis).

The product is the sm_100a shared library ``lib/libpawan_gpu.so`` behind the
C ABI of ``include/pawan_gpu.h``; ``capi`` binds it for Python, ``dropin/``
holds the C++ classes that plug it into PAWAN's ``__interaction`` /
``__integration`` surface, and ``cases`` generates the benchmark workloads.
"""
__version__ = "0.1.0"
