"""CPU oracle of the H2 matvec (test infrastructure; see oracle.py and h2oracle.c)."""
