"""swirlc_b200: B200-native Swirl-C compressible RHS + SSP-RK3 hot path.

Mirrors the module layout and call signatures of the reference's hot path
(swirl_c.equations, swirl_c.numerics, swirl_c.boundary, swirl_c.core) over
torch CUDA tensors; the arithmetic runs in the sm_100a kernels of
libswirlc_b200.so (include/swirlc_b200.h).
"""

__version__ = '0.1.0'
