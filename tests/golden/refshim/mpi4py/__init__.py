"""Single-rank stand-in for mpi4py (golden-vector generation only)."""
