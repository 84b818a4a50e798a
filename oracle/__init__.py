"""CPU oracle for the tracking path -- TEST INFRASTRUCTURE ONLY.

A plain-C restatement of HaissinskiJulia's longitudinal_evolve! turn loop
(oracle.c), used only by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg as the checker.  Parity status: unpinned against the reference
itself (no Julia here, no golden vectors in the reference); see oracle.h.
"""
from .pyoracle import Oracle, OracleState  # noqa: F401
