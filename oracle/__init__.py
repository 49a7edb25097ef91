"""CPU oracle for the uFEM linear static path (test infrastructure only)."""
