"""CPU oracle of the stargaze integrator — test infrastructure only.

Only the test suite, the smoke check and the CPU-baseline leg of the
benchmark import this package. It is never part of the product path.
"""
