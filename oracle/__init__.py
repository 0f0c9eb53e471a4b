"""CPU oracle for the TT-SVD / TR-SVD hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this module;
only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its CPU baseline
leg and its ``--impl reference`` arm) use it, and only as the FP64 reference the
CUDA results are compared with or as the timed CPU stand-in for the reference's
own CPU path.
"""
from .ttsvd_oracle import *  # noqa: F401,F403
