"""CPU oracle for the searchlight alignment path (TEST INFRASTRUCTURE ONLY).

ha_oracle: numpy restatement of the reference path; ref_lib: ctypes binding of
the reference C library compiled by oracle/Makefile into oracle/_ref/.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
