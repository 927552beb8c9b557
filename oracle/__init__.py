"""CPU checker for the gridder (test infrastructure only; see oracle.py)."""
