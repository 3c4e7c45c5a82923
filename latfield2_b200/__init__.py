"""latfield2_b200 -- B200 (sm_100a) particle-mesh path of LATfield2.

CIC deposits (scalar, vector and symmetric-tensor CIC-NGP, full-CIC vector
and VecVec), CIC gather with kick, drift and rebin of brick-binned particles,
and the PM grid operator (real-to-complex FFT and a Poisson force), written as
CUDA kernels behind the C ABI in include/lf2gpu.h.  `Context`, `FieldHandle`,
`KFieldHandle` and `SlabFFT` are the Python binding of that ABI;
include/latfield2_b200.hpp gives C++ code the reference's Lattice / Field /
Particles / projection names over it.
"""
from ._lib import (DEPOSIT_FIXED64, DEPOSIT_FP32, DEPOSIT_FP32_PLAIN, LF2Error, library_path,  # noqa: F401
                   load)
from .core import Context, FieldHandle, KFieldHandle, SlabFFT  # noqa: F401
