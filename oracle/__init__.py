"""The oracle: CPU restatement of empanada's read-overlap path (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, and only as the checker.  The product (empanada_b200) never imports it.
"""
