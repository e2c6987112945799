"""B200 collective-coordinate (CC) stealthy potential.

The product is the C ABI of ``libccgpu.so`` (``include/cc_gpu.h``): hand-written sm_100a kernels for
rho(k) = sum_j exp(i k.r_j), the energy sum_k V(k)|rho(k)|^2/Volume + Shift, the forces and S(k). This package is a
thin ctypes binding of that ABI for Python callers (tests, benchmarks); it mirrors the reference's ShiftedCCPotential
interface (Energy, AllForce, Force, GetRho, SetConfiguration) and has no CPU fallback.
"""
from .ccgpu import (PATH_AUTO, PATH_NUFFT, PATH_SPLIT, PREC_FP64, PREC_MIXED, PREC_SCHEDULE,
                    STOPVAL_GROUND_STATE, CCBatch, CCError, CCMulti, CCPotential, NotANumberFound, device_available,
                    isotropic_kset, isotropic_structure_factor, library_path, load_library, probe_fma_peak, serve,
                    stealthy_kset)

__all__ = ["PATH_AUTO", "PATH_NUFFT", "PATH_SPLIT", "PREC_FP64", "PREC_MIXED", "PREC_SCHEDULE",
           "STOPVAL_GROUND_STATE", "CCBatch", "CCError", "CCMulti", "CCPotential", "NotANumberFound",
           "device_available", "isotropic_kset", "isotropic_structure_factor", "library_path", "load_library",
           "probe_fma_peak", "serve", "stealthy_kset"]
