"""CPU oracle for the textured 2DGS path -- test infrastructure only.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg,
always as the checker; the product package never imports it.
"""
