"""ORACLE — test infrastructure only.

CPU restatement of the reference (SweSoe/Zebraflow) hot path.  The parity
tests in tests/ and ``__graft_entry__.smoke()`` compare the GPU path against
it, and the CPU baseline leg of ``bench.py`` times it.  The product library
never imports or links it.
"""
