"""ORACLE — test infrastructure only (checker and CPU reference arm), never product code.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this.
"""
