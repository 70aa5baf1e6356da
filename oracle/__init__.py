"""The oracle: test infrastructure that states what the reference computes.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this package, and only as the checker (or the timed CPU baseline). The
product (gjxl_b200/) never imports it.

Two parts:
  * ``ref``: the reference's own CPU analysis code, compiled from its sources
    by oracle/Makefile into oracle/_ref/libgjxl_ref.so, reached through the
    stage-level C shim in oracle/ref_shim.cpp;
  * ``restate``: numpy restatements of the reference's stage arithmetic, each
    citing the reference file:line it follows, checked against ``ref`` and the
    committed golden vectors.
"""
