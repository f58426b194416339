"""Physical constants of the reference (Src/main.f90:124-129,
Src/read_reactions.f90:96-99).

The legacy driver assigns ``qe=1.60217646e-19`` without a ``d0`` suffix, so
the Fortran value is the float32-rounded 1.6021764682116162e-19; the modular
driver (modules/core/mod_constants.f90:7) uses the exact double.  This package
fixes the exact double everywhere (oracle and GPU use the same value).
"""
QE = 1.60217646e-19          # C
C_LIGHT = 2.99792458e8       # m/s
EPS0 = 8.854187817e-12       # F/m
AMU = 1.66053886e-27         # kg
ME = 9.10938188e-31          # kg (electron mass, Src/read_reactions.f90:97)
KB = 1.3806504e-23           # J/K, only used to turn a gas pressure into ngas
PI = 3.141592653589793       # 4 atan(1)
