"""CPU oracle of the AnDFN solve (test infrastructure only; see oracle.py)."""
