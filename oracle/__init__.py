"""CPU oracle of the FASES solver hot path -- TEST INFRASTRUCTURE ONLY.

fz_oracle.cpp restates the reference update loop in FP64; build.py compiles it; oracle.py is its
ctypes front end; build_ref.sh builds the reference solver itself from its own sources (into
oracle/_ref/) so that the restatement can be pinned against it. Nothing in the product imports
this package.
"""
