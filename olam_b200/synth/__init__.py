"""Synthetic inputs (grid and atmospheric states) for tests and benchmarks."""
