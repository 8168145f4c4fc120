"""Package data (bundled substitution matrices)."""
