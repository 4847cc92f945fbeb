"""Comparison helpers for the GPU parity tests (tolerances are stated where used)."""
import numpy as np


def rel_rms(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.sqrt(np.mean(b * b))
    num = np.sqrt(np.mean((a - b) ** 2))
    return num / den if den > 0 else num


def rel_err(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def energy_scale(s):
    """Coulomb magnitude sum_{i<j} |q_i q_j| / r_ij (minimum image for PME), the
    scale against which an energy error is judged when the total cancels."""
    p = np.asarray(s.positions, dtype=np.float64)
    q = np.abs(np.asarray(s.charges, dtype=np.float64))
    d = p[None, :, :] - p[:, None, :]
    if s.method == 1:
        box = np.asarray(s.box, dtype=np.float64)
        d -= box * np.floor(d / box + 0.5)
    r = np.sqrt((d * d).sum(-1))
    iu = np.triu_indices(len(q), 1)
    return float((q[:, None] * q[None, :])[iu] @ (1.0 / r[iu]))


def energy_rms_scale(s):
    """sqrt(sum_{i<j} (q_i q_j / r_ij)^2): rounding errors of the pair terms
    (relative ~6e-8 each in FP32) add in quadrature on this scale."""
    p = np.asarray(s.positions, dtype=np.float64)
    q = np.asarray(s.charges, dtype=np.float64)
    d = p[None, :, :] - p[:, None, :]
    if s.method == 1:
        box = np.asarray(s.box, dtype=np.float64)
        d -= box * np.floor(d / box + 0.5)
    r = np.sqrt((d * d).sum(-1))
    iu = np.triu_indices(len(q), 1)
    e = (q[:, None] * q[None, :])[iu] / r[iu]
    return float(np.sqrt(e @ e))
