"""lens_sensor_b200: B200-native FDTD time stepping for the lens_sensor waveguide sensor.

Hot path: 2D TE/TM and 3D Yee CPML leapfrog with loss, sub-pixel bead
permittivity, Huygens CW source and steady-state DFT phasors, run by
hand-written sm_100a kernels behind the C ABI in include/lens_fdtd.h.
"""
__version__ = '0.1.0'
