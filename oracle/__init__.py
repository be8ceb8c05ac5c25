"""CPU oracle for the Dirac-operator hot path (test infrastructure only)."""
