"""Command-line drivers (the reference's simulation_toolkit/cli)."""
