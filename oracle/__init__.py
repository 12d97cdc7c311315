"""CPU oracle of the MHIT36 timestep (TEST INFRASTRUCTURE ONLY).

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, as the
checker.  The product (mhit36_mixedp_b200) never imports it.
"""
