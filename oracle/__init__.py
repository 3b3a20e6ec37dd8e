"""CPU oracle for the trace-commitment path (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this package, and only as the checker or the timed CPU baseline.
"""
