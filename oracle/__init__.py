"""CPU oracle of JuMC's electron step -- TEST INFRASTRUCTURE.

Imported only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm.  Parity against the Julia reference is unpinned (see oracle.h).
"""
