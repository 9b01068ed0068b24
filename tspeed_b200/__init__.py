"""tspeed_b200: B200 (sm_100a) engine for tspeed's explicit leap-frog loop.

The compute lives in libtspeed_b200.so (CUDA kernels behind a C-ABI,
include/tspeed_b200.h). `tspeed_b200.capi.Simulation` is the Python face of
one engine handle; `tspeed_b200.workloads` builds the seeded benchmark
problems.
"""
__all__ = ["capi", "workloads"]
