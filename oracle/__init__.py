"""ORACLE — test infrastructure only.

CPU restatement of the reference (SweSoe/Zebraflow) hot path, that the parity
tests compare against, in tests/, by ``__graft_entry__.smoke()`` and by the CPU
baseline leg of ``bench.py``.  The product library never imports or links it.
"""
