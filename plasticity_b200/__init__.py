"""B200-native crystal-plasticity quadrature-point hot path.

A drop-in for PRISMS-Plasticity's per-qp constitutive update
(calculatePlasticity), its algorithmic tangent and the element
residual/stiffness contraction (getElementalValues), exposed as a C ABI
(include/cp_gpu.h) implemented by hand-written sm_100a CUDA kernels in
csrc/.  ``capi.CpHandle`` is the Python view of that ABI; ``harness`` is a
host Newton loop that calls it the way the reference's ellipticBVP does.
"""
from .capi import CpError, CpHandle, CpMaterial, CpOptions, default_options, load_library  # noqa: F401
