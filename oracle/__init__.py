"""CPU parity oracle for the garli_b200 engine (test infrastructure only)."""
