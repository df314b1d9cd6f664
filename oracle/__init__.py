"""Oracle package (test infrastructure only).

CPU FP64 restatement of the reference's patch-advance path. Only tests/,
__graft_entry__.smoke() and the CPU-baseline leg of bench.py load it; the
product (amrclaw_b200) never does.
"""
