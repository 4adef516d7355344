"""CPU FP64 oracle of the spherical-transform cycle -- test infrastructure only."""
