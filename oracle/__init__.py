"""CPU oracle for the onion-gen key-search hot path (test infrastructure only)."""
