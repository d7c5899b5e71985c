"""Where the reference checkout lies -- TEST INFRASTRUCTURE ONLY.

The reference (alvarospace/hpc_ode) is read only to build the checker (its
pyJac C chemistry, oracle/Makefile ``ref``) and to generate golden fixtures; the
GPU path never reads it.  Its location comes from the environment variable
HPC_ODE_REFERENCE, else from the ``reference_path`` key of BASELINE.json at the
repository root; None when neither names an existing directory.
"""
from __future__ import annotations

import json
import os
from typing import Optional

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference_dir() -> Optional[str]:
    cand = os.environ.get("HPC_ODE_REFERENCE")
    if not cand:
        try:
            with open(os.path.join(ROOT, "BASELINE.json")) as f:
                cand = json.load(f).get("reference_path")
        except (OSError, ValueError):
            cand = None
    return cand if cand and os.path.isdir(cand) else None


def reference_subdir(*parts: str) -> Optional[str]:
    """A directory inside the reference checkout, or None when it is absent."""
    base = reference_dir()
    if base is None:
        return None
    p = os.path.join(base, *parts)
    return p if os.path.isdir(p) else None
