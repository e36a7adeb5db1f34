"""The reference's own step kernels compiled for the host CPU (test infrastructure only)."""
