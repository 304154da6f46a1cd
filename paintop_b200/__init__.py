"""paintop_b200 -- the B200 `cuda` backend of paintop's Poisson / screened-Poisson ops.

The compute path is ``libpaintop_cuda.so`` (hand-written sm_100a kernels behind
the C ABI in include/paintop_cuda.h); this package holds its build script, the
ctypes binding, the Python face of the ops and the seeded workload generators.
"""
__all__ = ["ops", "synth", "build"]
