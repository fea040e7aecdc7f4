"""B200-native PatchStereo depth-map engine (drop-in for the cumulus3d PatchMatch backend).

The engine is ``libpatchstereo.so`` (CUDA kernels for sm_100a + a C++ runtime behind the C ABI in
``include/patchstereo.h``).  This package holds its sources (``csrc/``), the build script, the Python mirror of the
reference's backend interface (``patchstereo``), the multi-scale driver (``densify``) and the synthetic workloads
(``scenes``).
"""
__all__ = ["patchstereo", "scenes", "densify", "build"]
