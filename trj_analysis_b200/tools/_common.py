"""Shared plumbing of the command-line tools."""
from __future__ import annotations

import os
import sys


def ensure_importable() -> None:
    """Lets the tools run as plain scripts (python path/to/tool.py traj.nc)."""
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    if root not in sys.path:
        sys.path.insert(0, root)


def species_of(types, nsp_hint=None):
    """Species numbering of a trajectory's type ids by first appearance (all types selected)."""
    import numpy as np
    from trj_analysis_b200 import refsem
    uniq = sorted(set(int(t) for t in np.unique(types)))
    sp, wtypes, _ = refsem.species_by_first_appearance(types, uniq)
    return sp, wtypes
