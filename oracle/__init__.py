"""Test-side checkers (FP64 oracle and the reference built from its own sources).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.
"""
