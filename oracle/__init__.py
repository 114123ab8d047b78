"""CPU oracle of the registration chain (test infrastructure only).

s2s3.py restates the reference's NumPy S2/S3 path; stitch_oracle.c restates
its S4 and S5 CUDA stages in plain C (built into liboracle.so by the
Makefile); chain.py runs the whole per-pair chain on the CPU. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use this package.
"""
