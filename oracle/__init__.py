"""Test infrastructure: CPU oracle for libbirdwing's multiply path.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this package; the product path never does.
"""
