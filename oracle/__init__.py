"""Test infrastructure: the CPU oracle for the colored BFM sweep.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg and
reference arm use this package.  The product (pscbfm_b200) never imports it.
"""
