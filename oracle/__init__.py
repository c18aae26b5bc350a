"""CPU oracle of the reference GROG path (test infrastructure only).

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, as the checker; the product never imports it.
"""
