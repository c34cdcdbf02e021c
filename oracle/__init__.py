"""ORACLE (test infrastructure): CPU restatement of the reference's passes.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, as the checker. Nothing in restir_b200 imports it.
"""
