"""CPU oracle of the Quantum++ hot path -- test infrastructure only.

Imported by tests/, by __graft_entry__.smoke() as the checker and by the
CPU-baseline leg of bench.py; never by the product package qpp_b200.
"""
