"""CPU restatement of the reference's Monte Carlo docking path (test infrastructure only)."""
