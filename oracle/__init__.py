"""Oracle — TEST INFRASTRUCTURE ONLY.

CPU restatements of the reference's algorithm (walk_oracle.c, cells_oracle.py)
and the recipes that build the reference's own code for the CPU as a checker
(build.py, refshim/, fake_pycuda.py).  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline legs use it; the product (nozomi_b200) never
imports it.
"""
