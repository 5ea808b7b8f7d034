"""Oracle package: CPU checker of the CUDA path (test infrastructure only)."""
