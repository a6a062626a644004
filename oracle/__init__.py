"""CPU restatement of MCM's explicit SPH step: TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, and only as the checker (or the timed CPU baseline).  Parity status:
unpinned (the reference has no tests, golden vectors or Fortran compiler here).
"""
