"""Test infrastructure: the CPU oracle for the DC forward + adjoint path.

Only `tests/`, `__graft_entry__.smoke()` and the CPU-baseline leg of
`bench.py` may import this package.  It is the checker, never part of the
product path.
"""
