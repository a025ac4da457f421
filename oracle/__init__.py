"""CPU oracle for the CudaKpz hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs
may import this package; it is the checker, never the product.
"""
