"""Phase timing of the batched energy path (CUDA events inside the engine)."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check


def phase_times(engine, ham, theta, repeats: int = 3, stream=None):
    """Median phase times (ms) of ``repeats`` profiled calls and launches per call."""
    from .engine import _ptr, _stream
    t = engine._theta(theta)
    B = t.shape[0]
    rows = []
    launches = ctypes.c_int()
    for _ in range(repeats):
        ms = (ctypes.c_double * 4)()
        check(engine.ctx, engine.lib.vqemps_profile_energy(engine.ctx, ham.handle, _ptr(t), B, ms,
                                                           ctypes.byref(launches), _stream(stream)),
              "profile_energy")
        rows.append(list(ms))
    med = np.median(np.array(rows), axis=0)
    names = ("prepare", "right_env", "levels", "reduce")
    return dict(ms=dict(zip(names, [float(v) for v in med])), levels_s=float(med[2]) * 1e-3,
                launches_per_step=launches.value)
