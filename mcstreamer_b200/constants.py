"""Physical constants used on the hot path (values of JuMC/src/constants.jl:50-54,149-150,
scipy 2014 CODATA set as shipped by the reference)."""

elementary_charge = 1.6021766208e-19
eV = 1.6021766208e-19
electron_mass = 9.10938356e-31
epsilon_0 = 8.854187817620389e-12
speed_of_light = 299792458.0
centi = 0.01
Td = 1e-21
nair = 2.6867811e25
