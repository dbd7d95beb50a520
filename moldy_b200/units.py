"""Model units of the MOLDY reference (src/constants_m.F90:84-113).

Energy eV, length Angstrom, mass amu; one model time unit is
sqrt(amu * A^2 / eV) = 1.018050530893617e-14 s; one model pressure unit is
eV/A^3 = 160.2176 GPa.
"""
AVOGADRO = 6.02214179e23
ELECTRON = 1.602176487e-19
ANGSTROM = 1.0e-10
BOLTZMANN = 1.3806504e-23
BK = BOLTZMANN / ELECTRON                      # eV per kelvin
TIME_TO_SEC = 1.018050530893617e-14
TIME_TO_FS = TIME_TO_SEC / 1.0e-15
FS_TO_TIME = 1.0 / TIME_TO_FS
PRESS_TO_GPA = (ELECTRON / ANGSTROM ** 3) / 1.0e9
GPA_TO_PRESS = 1.0 / PRESS_TO_GPA
FE_MASS = 55.845                               # src/particles_m.F90 reference mass of Fe
