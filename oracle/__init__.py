"""CPU oracle for the CDT path: test infrastructure only (see oracle.py)."""
