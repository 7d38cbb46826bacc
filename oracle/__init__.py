"""CPU FP64 oracle for the AMOEBA energy/gradient path (test infrastructure only)."""
