"""CPU oracle for the PDHG path (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package; the product never does.
"""
