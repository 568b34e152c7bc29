"""ORACLE -- test infrastructure only.

CPU restatements (and, in this container, shims that let the unmodified
reference package run) used as the checker by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The product
package ``polyspec_b200`` never imports anything from here.
"""
