"""TEST INFRASTRUCTURE ONLY: the CPU oracle for VirtualCBCT's hot paths.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm may import this package, and only as the checker.  The product
package ``virtualcbct_b200`` never imports it.

Two kinds of oracle live here:

* ``liboracle.so`` -- a double-precision restatement of the reference's
  arithmetic (``vcbct_oracle.c``), bitwise faithful to the reference where the
  reference is deterministic;
* ``_ref/libref_proj.so`` / ``_ref/libref_fdk.so`` -- the reference's own CPU
  code (``Release_CBCT_Projection_CM/reprojection.cpp`` etc.) compiled from its
  sources by ``oracle/Makefile``, used to pin the restatement and as the timed
  CPU baseline.
"""
from .oracle import *  # noqa: F401,F403
