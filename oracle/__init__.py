"""The oracle: CPU restatement of the reference scan path (test infrastructure only)."""
