"""CPU oracle for the star-query hot path — test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs use it.
"""
