"""Where the reference checkout lies -- TEST INFRASTRUCTURE ONLY.

The reference (alvarospace/hpc_ode) is read only to build the oracle's
reference kernels (its pyJac C chemistry, oracle/Makefile ``ref``) and to generate golden fixtures; the
GPU path never reads it.  Its location comes from the environment variable
HPC_ODE_REFERENCE, else the checkout's default location (DEFAULT_REFERENCE);
None when neither is an existing directory.
"""
from __future__ import annotations

import os
from typing import Optional

DEFAULT_REFERENCE = "/root/reference"


def reference_dir() -> Optional[str]:
    cand = os.environ.get("HPC_ODE_REFERENCE") or DEFAULT_REFERENCE
    return cand if os.path.isdir(cand) else None


def reference_subdir(*parts: str) -> Optional[str]:
    """A directory inside the reference checkout, or None when it is absent."""
    base = reference_dir()
    if base is None:
        return None
    p = os.path.join(base, *parts)
    return p if os.path.isdir(p) else None
