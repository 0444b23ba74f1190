"""SI units and constants with the values of include/crpropa/Units.h."""
import math

meter = 1.0
second = 1.0
kilogram = 1.0
ampere = 1.0
newton = 1 * kilogram * meter / second / second
joule = 1 * newton * meter
tesla = 1 * newton / ampere / meter
volt = 1 * kilogram * meter * meter / ampere / second / second / second
coulomb = 1 * ampere * second

eplus = 1.602176487e-19 * ampere * second
c_light = 2.99792458e8 * meter / second
c_squared = c_light * c_light
amu = 1.660538921e-27 * kilogram
mass_proton = 1.67262158e-27 * kilogram
mass_electron = 9.10938291e-31 * kilogram

gauss = 1e-4 * tesla
microgauss = 1e-6 * gauss
nanogauss = 1e-9 * gauss
muG = microgauss
nG = nanogauss

electronvolt = eplus * volt
eV = electronvolt
keV = 1e3 * eV
MeV = 1e6 * eV
GeV = 1e9 * eV
TeV = 1e12 * eV
PeV = 1e15 * eV
EeV = 1e18 * eV

au = 149597870700 * meter
ly = 365.25 * 24 * 3600 * second * c_light
parsec = 648000 / math.pi * au
kiloparsec = 1e3 * parsec
megaparsec = 1e6 * parsec
gigaparsec = 1e9 * parsec
pc = parsec
kpc = kiloparsec
Mpc = megaparsec
Gpc = gigaparsec

kilometer = 1000 * meter
km = kilometer
year = 365.25 * 24 * 3600 * second
Myr = 1e6 * year
Gyr = 1e9 * year
