"""B200-native spherical-transform cycle (Calypso sph_b_trans / sph_f_trans path)."""
from .config import SphConfig, CFG1, CFG2, CFG3, CFG5, NAMED  # noqa: F401
