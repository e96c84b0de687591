"""CPU oracle of the walk (test infrastructure only; see oracle.py)."""
