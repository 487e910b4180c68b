"""CPU FP64 oracle of the solve path (test infrastructure only)."""
