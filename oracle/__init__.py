"""Test-side checkers (FP64 oracle and the reference built from its own sources).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.

REFERENCE is where the reference checkout is read from when the checkers are built:
the environment variable SKM_REFERENCE, with its default set here and nowhere else.
Nothing reads it at run time on a machine without the checkout.
"""
import os

REFERENCE = os.environ.get("SKM_REFERENCE", "/root/reference")
