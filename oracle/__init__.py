"""TEST INFRASTRUCTURE ONLY: CPU oracles for the B200 search path.

  oracle.ref   -- the reference engine itself, compiled from its sources by
                  oracle/Makefile into oracle/_ref/ (FP32 and FP64 builds)
  oracle.port  -- dmst_oracle.c, a plain-C restatement of the same algorithm

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, and only as the checker or the timed CPU baseline -- never as part
of the product path.
"""
