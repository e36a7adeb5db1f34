"""Helpers shared by the GPU parity tests (CUDA path vs the CPU oracle)."""
from __future__ import annotations

import numpy as np

STATE_FIELDS = ["ETA1", "ETA2", "NODE_Z", "NODE_U2", "NODE_W2", "NODE_TR", "NODE_KB", "NODE_DRY",
                "SIDE_U2", "SIDE_BTU", "SIDE_ZC", "SIDE_KB", "SIDE_DRY", "SIDE_U", "SIDE_HHAT", "SIDE_CHI",
                "SIDE_QH", "SIDE_GRADETA1", "SIDE_GRADETA2",
                "ELEM_Z", "ELEM_W", "ELEM_QV", "ELEM_TR", "ELEM_KB", "ELEM_DRY", "ELEM_GHAT",
                "JCG_X", "JCG_X1", "JCG_X2", "ELBC"]


def copy_state(oracle, model, member: int = 0) -> None:
    """Put every exchangeable field of the oracle into the GPU member (reference numbering)."""
    for f in STATE_FIELDS:
        model.put(member, f, oracle.get(f))


def relerr(a, b, mask=None) -> float:
    """Norm-wise relative difference max|a-b| / max|b| (0 when both are zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
    if a.size == 0:
        return 0.0
    scale = np.abs(b).max()
    d = np.abs(a - b).max()
    return float(d / scale) if scale > 0 else float(d)


def level_mask(kb: np.ndarray, nvrt: int) -> np.ndarray:
    """[nvrt, n] mask of levels at or above each entity's bottom level."""
    return np.arange(nvrt)[:, None] >= kb[None, :]
