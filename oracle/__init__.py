"""CPU oracle of the warpflow-les hot path (test infrastructure only)."""
