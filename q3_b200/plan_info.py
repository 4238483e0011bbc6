"""Host-side facts about a k-point's sticks layout (for reporting and sizing)."""
from __future__ import annotations

import numpy as np


def stick_count(kp, grid) -> int:
    """Distinct (w1, w2) grid columns holding at least one G of the sphere."""
    n1, n2, n3 = grid
    f = kp.g_to_grid[kp.g_to_grid >= 0].astype(np.int64)
    return int(np.unique(f // n3).size)


def row_count(kp, grid) -> int:
    """Distinct w1 among the sticks."""
    n1, n2, n3 = grid
    f = kp.g_to_grid[kp.g_to_grid >= 0].astype(np.int64)
    return int(np.unique(f // (n2 * n3)).size)
