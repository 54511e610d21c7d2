"""B200 (sm_100a) direct spherical Biot-Savart sum and RK4 driver for ThesisCode's
barotropic-vorticity panel method.

The compute path is libthesiscode_b200.so (CUDA kernels behind the C ABI of
include/thesiscode_b200.h); this package holds its ctypes binding and the host
mirror of the reference's module interfaces.
"""
__version__ = "0.1.0"
