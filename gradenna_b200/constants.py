"""Physical constants in SI units (same values as src/gradenna/constants.py:3-6)."""

C0 = 299792458.0  # speed of light in vacuum [m/s]
MU0 = 1.25663706212e-06  # vacuum permeability [H/m]
EPS0 = 1.0 / (MU0 * C0**2)  # vacuum permittivity [F/m]
ETA0 = MU0 * C0  # impedance of free space [ohm]
