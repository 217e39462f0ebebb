"""CPU checkers (test infrastructure; see oracle.py)."""
