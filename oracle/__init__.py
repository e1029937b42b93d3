"""TEST INFRASTRUCTURE ONLY.

The oracle for the RCA beamformer: a CPU restatement of the reference
arithmetic (rca_oracle.c, fp64.py, host.py) and the reference kernel itself
built from its own source (Makefile -> _ref/).  Only tests/,
__graft_entry__.smoke() and bench.py's accuracy / CPU-baseline legs use it,
and only as the checker; the product (simu_rca_ab_b200, librcabf) never
imports, links or calls anything here.
"""
