"""TEST INFRASTRUCTURE — the parity oracle.

* ``oracle.qkoracle``: the CPU restatement of the reference algorithm
  (``oracle/qk_oracle.c``), driven by the engine's Philox counters.
* ``oracle.qkref``: the reference's own headers compiled against a host shim
  (``oracle/ref_harness``, outputs in ``oracle/_ref``).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference
arm import this package, as the checker; the engine never does.
"""
