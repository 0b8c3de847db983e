"""Test infrastructure (the oracle): the C restatement of the reference kernels
and the recipe that compiles the reference itself.  Only tests/, smoke() and
bench.py's CPU-baseline leg import this package."""
