"""Test-only checker: FP64 CPU oracle and the reference-kernel launcher.

Nothing in the product (sapporo2_b200/) imports this package; only tests/,
the smoke check and the CPU-baseline leg of bench.py do.
"""
