"""phx: B200-native (sm_100a) per-iteration hot path of PHengLEI's unstructured
NS / Spalart-Allmaras solver behind a C ABI (include/phx.h).

Modules: ``solver`` (ctypes front end mirroring NSSolverUnstruct), ``mesh``
(synthetic grids in the reference's face layout), ``cases`` (benchmark cases),
``build`` (nvcc build of libphx.so).
"""
