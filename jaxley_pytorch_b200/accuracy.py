"""Float32 accuracy against float64: the voltage error over the non-chaotic stretches
of a trace, where the 1e-3 mV bar applies, and over the whole trace.

A spike amplifies any rounding difference into a shift of its timing, so over a
spiking stretch a float32 run and a float64 run of the same model differ by the
voltage slope times the shift (mV-scale near the upstroke) without either being
wrong. The subthreshold stretches are the samples below -50 mV with no sample above
-20 mV (a spike) in the preceding 5 ms (200 steps of 0.025 ms), judged on the
float64 trace."""
from __future__ import annotations

from typing import Dict, Optional, Sequence

import numpy as np

SPIKE_MV = -20.0
SUBTHRESHOLD_MV = -50.0
WINDOW_STEPS = 200


def subthreshold_mask(v64: np.ndarray, window: int = WINDOW_STEPS) -> np.ndarray:
    """Boolean mask of the subthreshold samples of float64 voltage traces
    `(..., time)` (see the module docstring)."""
    v64 = np.asarray(v64)
    spk = (v64 > SPIKE_MV).astype(np.int64)
    c = np.cumsum(spk, axis=-1)
    lag = np.zeros_like(c)
    if c.shape[-1] > window:
        lag[..., window:] = c[..., :-window]
    recent = (c - lag) > 0
    return (v64 < SUBTHRESHOLD_MV) & ~recent


def voltage_errors(v64: np.ndarray, v32: np.ndarray) -> Dict[str, Optional[float]]:
    """max |v32 - v64| in mV over the whole traces and over their subthreshold
    stretches, and the fraction of subthreshold samples."""
    d = np.abs(np.asarray(v32, dtype=np.float64) - np.asarray(v64, dtype=np.float64))
    sub = subthreshold_mask(v64)
    return {"max_dv_mV": float(d.max()),
            "max_dv_subthreshold_mV": float(d[sub].max()) if sub.any() else None,
            "subthreshold_fraction": float(sub.mean()),
            "spiking": bool((np.asarray(v64) > SPIKE_MV).any())}


def gradient_error(g64: np.ndarray, g32: np.ndarray) -> float:
    """Largest deviation of a float32 gradient over the largest float64 entry."""
    g64 = np.asarray(g64, dtype=np.float64)
    return float(np.abs(np.asarray(g32, dtype=np.float64) - g64).max() / max(np.abs(g64).max(), 1e-300))


def voltage_columns(recordings: Sequence) -> list:
    """Columns of the voltage recordings among `(name, node)` recordings."""
    return [c for c, (name, _) in enumerate(recordings) if name == "v"]
