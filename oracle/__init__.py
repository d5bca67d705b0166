"""CPU FP64 oracle of the aperi-mech hot path (test infrastructure only)."""
