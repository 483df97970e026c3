"""rspacedist_b200 -- B200 (sm_100a) implementation of RSPACE kukan's
real-space Kohn-Sham hot path behind a C ABI (include/rspace_b200.h).

Modules:
  lib     -- ctypes binding of librspace_b200.so (fails loudly if missing)
  build   -- nvcc build of the library (sm_100a, in-tree)
  system  -- host set-up of cells: grid, atoms, sphere lists, projectors
  kukan   -- the kukan-named entry points on torch CUDA tensors
"""
__version__ = "0.1.0"
