"""CPU oracle and reference cross-check build (test infrastructure only)."""
