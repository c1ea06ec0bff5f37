"""tclb_b200: a B200-native lattice-Boltzmann engine for TCLB's Run path."""
from . import models  # noqa: F401
