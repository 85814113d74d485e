"""CPU oracle for the MPM hot path (test infrastructure only).

`oracle.lib` wraps two kinds of CPU code:
  * liboracle.so -- this repository's serial restatement of the reference
    algorithm (oracle/dmpm_oracle.cpp), FP32 and FP64;
  * oracle/_ref/libref_fp{32,64}.so -- the reference's own sources compiled
    here by oracle/build_ref.sh (present only where the reference was).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""
