"""Solver drivers (drop-in for the reference's src/solvers package)."""
