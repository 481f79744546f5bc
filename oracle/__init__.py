"""ORACLE — test infrastructure only (CPU checkers of the CUDA library)."""
