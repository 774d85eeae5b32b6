"""ORACLE (test infrastructure only): float64 restatement of the reference's
seasonal forcing blend, ``interp_monthly_field_jit``
(src/zhenmode/model/inputs/forcing/seasonal.py:86-103).  Only ``tests/``
import it; pinned against ``tests/golden/seasonal_blend.npz``."""
from __future__ import annotations

import numpy as np


def blend(stack, day, blend_days=5.0):
    month_len = 30.0
    mpos = day % month_len
    mi = int(np.floor(day / month_len)) % 12
    prev_i, nxt_i = (mi - 1) % 12, (mi + 1) % 12
    if blend_days <= 0.0:
        return np.asarray(stack[mi], dtype=np.float64)
    half = blend_days / 2.0
    w_after = min(max((mpos - (month_len - half)) / blend_days, 0.0), 1.0)
    w_before = min(max((half - mpos) / blend_days, 0.0), 1.0)
    s = np.asarray(stack, dtype=np.float64)
    return (1.0 - w_after - w_before) * s[mi] + w_after * s[nxt_i] + w_before * s[prev_i]
