"""CPU oracle for the MPS VQE hot path (test infrastructure; never the product path)."""
