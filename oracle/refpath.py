"""TEST INFRASTRUCTURE ONLY: where the reference source tree is read from.

The reference checkout is only read on the development machine (to build
``oracle/_ref`` and to regenerate fixtures); GPU test runs use the prebuilt
``oracle/_ref`` files and the committed fixtures instead.  One lookup order
for every script and test, the same as ``oracle/Makefile``'s ``REF``:

1. the environment variable ``VCBCT_REFERENCE``;
2. ``baseline/_ref`` at the repository root, where present;
3. the read-only checkout at ``/root/reference``.
"""
from __future__ import annotations

import os

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
_CHECKOUT = "/root/reference"


def reference_root() -> str:
    env = os.environ.get("VCBCT_REFERENCE")
    if env:
        return env
    local = os.path.join(ROOT, "baseline", "_ref")
    if os.path.isdir(os.path.join(local, "Release_CBCT_Projection_CM")):
        return local
    return _CHECKOUT


def reference_path(*parts: str) -> str:
    """A path inside the reference tree (it may not exist on a GPU host)."""
    return os.path.join(reference_root(), *parts)
