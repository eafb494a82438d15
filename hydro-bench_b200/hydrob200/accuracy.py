"""Error measures of a reduced-precision state against an fp64 state.

A depth error is reported two ways over the wet cells (reference depth above
HM2, the threshold below which the reference clips velocities,
functors.cu:759-762):
  rel_max   max_i |H_i - Hr_i| / Hr_i, the largest per-cell relative error;
  normwise  max_i |H_i - Hr_i| / max_i Hr_i.
The mass error is the relative change of sum(H * AREA) over all cells.
"""
from typing import Dict

import numpy as np


def depth_error(h: np.ndarray, h_ref: np.ndarray, hm2: float, area: np.ndarray = None) -> Dict[str, float]:
    h = np.asarray(h, np.float64)
    h_ref = np.asarray(h_ref, np.float64)
    wet = h_ref > hm2
    d = np.abs(h - h_ref)
    out = {
        "rel_max": float(np.max(d[wet] / h_ref[wet])) if wet.any() else 0.0,
        "normwise": float(np.max(d[wet]) / np.max(h_ref[wet])) if wet.any() else 0.0,
        "wet_cells": int(wet.sum()),
    }
    if area is not None:
        a = np.asarray(area, np.float64)
        out["mass_rel"] = float(np.sum(h * a) / np.sum(h_ref * a) - 1.0)
    return out
