"""CPU checker for natinterp3d_b200 -- test infrastructure only.

The C restatement of natinterp3d's query path (``nif_oracle.c``) and natinterp3d's
own query code compiled from its sources (``_ref``).  Only tests, the smoke
check and bench.py's CPU-baseline leg use this package.
"""
