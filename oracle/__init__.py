"""CPU oracle for the IFGF matvec: test infrastructure only (see oracle.py)."""
