"""B200-native (sm_100a) engine for the XFDTD_CORE 3-D FDTD time step.

* ``engine``  -- ctypes binding of the C ABI in include/xfd_engine.h
* ``host``    -- ctypes binding of the C++20 host library (xfdtd::Simulation)
* ``scene``   -- scene descriptions and the benchmark workloads
* ``build``   -- in-tree build of the native libraries
"""
__all__ = ["engine", "scene", "build"]
