"""CPU oracle for the separable-convolution path (test infrastructure only)."""
