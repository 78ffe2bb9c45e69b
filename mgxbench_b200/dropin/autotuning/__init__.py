"""MGXBench's `autotuning` package, as this library replaces it (see predictive.py)."""
