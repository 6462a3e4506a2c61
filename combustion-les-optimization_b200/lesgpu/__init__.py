"""B200-native LES combustion solver step (host side).

The CUDA step kernels live in ``liblesgpu.so`` (built from ``csrc/``) behind the C ABI in
``include/les_gpu.h``; this package is the Python mirror of the solver's host loop.
"""
