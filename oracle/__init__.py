"""CPU FP64 oracle package: test infrastructure only (see oracle.py)."""
