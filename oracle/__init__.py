"""CPU oracle for the FastRRT planning hot path (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package; the product package fastrrt_b200 never does.
"""
