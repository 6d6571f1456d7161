"""Error measures of a run against an FP64 run of the same input: relative
L1 (sum |a - b| / sum |b|) and Linf (max |a - b|, absolute and relative to
max |b|) of the interior density and total energy."""
from __future__ import annotations

import numpy as np

VARS = {"rho": 0, "E": 3}


def field_errors(a: np.ndarray, b: np.ndarray) -> dict:
    out = {}
    for name, v in VARS.items():
        x = a[v, 2:-2, 2:-2].astype(np.float64)
        y = b[v, 2:-2, 2:-2].astype(np.float64)
        d = np.abs(x - y)
        out[name] = {"l1_rel": float(d.sum() / np.abs(y).sum()),
                     "linf_abs": float(d.max()),
                     "linf_rel": float(d.max() / np.abs(y).max())}
    return out
