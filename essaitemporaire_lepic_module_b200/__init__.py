"""B200-native (sm_100a) hot path of the LePIC 3D PIC-MCC timestep.

Modules:
  config     synthetic workloads and the constants the reference derives
  geometry   wall-label mask and Dirichlet potential (generate_boundary)
  reactions  chemistry files and cross-section tables (read_reactions)
  dropin     Python mirror of the reference routines over the C-ABI drop-ins
  sim        device-resident time stepping through the device API
  build      nvcc build of liblepic_gpu.so (sm_100a)
"""
__all__ = ["config", "geometry", "reactions", "dropin", "sim", "build"]
