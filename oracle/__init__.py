"""CPU oracle of the FUGU-2D hot path -- test infrastructure only (the checker).

Only tests/, __graft_entry__.smoke() and the CPU legs of bench.py import this
package; the product never does.
"""
