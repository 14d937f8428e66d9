"""CPU oracle of the MRPNN cloud-rendering path -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
may import this package; the product (internship_b200) never does.
"""
