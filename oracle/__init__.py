"""ORACLE -- test infrastructure only.

CPU restatements of the reference's Eq. (C7) path (exmarg/search/*.py), used as the
checker by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline and reference
legs.  The exmarg_b200 package never imports anything from here.
"""
