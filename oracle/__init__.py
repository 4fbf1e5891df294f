"""CPU oracle of the massively primitive path (test infrastructure only)."""
