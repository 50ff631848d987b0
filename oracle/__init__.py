"""CPU oracle of the AVISM hot path -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, as the checker.  The product (avism_b200) never imports it.
"""
