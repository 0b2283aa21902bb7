"""CPU oracle of the elliptic solve path (test infrastructure only)."""
