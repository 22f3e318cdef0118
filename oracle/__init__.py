"""CPU oracle of the HIT_Solver hot path: test infrastructure only."""
