"""idcsweep: B200-native 2-D upwind-DG transport sweep (the hot path of crockatt/idc-transport-solver).

* ``abi``        ctypes binding of the C ABI (include/idcsweep.h, libidcsweep.so)
* ``quadrature`` level-symmetric S_N ordinate sets in the reference's quadrant order
* ``problems``   seeded synthetic problems of the benchmark shapes (lattice, log-normal)
"""
