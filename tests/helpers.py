"""Shared helpers for the tests: seeded inputs and comparisons."""
import numpy as np

import oracle as O


def consistent(shell: "O.Shell", v):
    """Copy the owner's value onto every duplicate (an assembled vector)."""
    v = np.array(v, dtype=np.float64, copy=True)
    cls = shell.classes.reshape(-1)
    own = shell.owned_lat.reshape(-1).astype(bool)
    lead = {}
    idx = np.where(cls >= 0)[0]
    for i in idx:
        if own[i]:
            lead[cls[i]] = i
    src = np.array([lead[cls[i]] for i in idx])
    if v.ndim == 4:
        flat = v.reshape(-1, shell.nr)
        flat[idx] = flat[src]
    else:
        for c in range(v.shape[0]):
            flat = v[c].reshape(-1, shell.nr)
            flat[idx] = flat[src]
    return v


def smooth_viscosity(shell: "O.Shell", seed: int, contrast: float = 10.0):
    """exp of a smooth random field on the shell (positive, nodal)."""
    rng = np.random.default_rng(seed)
    X = shell.physical_coords()
    f = np.zeros(X.shape[:-1])
    for _ in range(6):
        kvec = rng.normal(size=3) * 3.0
        ph = rng.uniform(0, 2 * np.pi)
        f += np.sin(X @ kvec + ph)
    f /= np.abs(f).max()
    return np.exp(np.log(contrast) * 0.5 * f)


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


BC_COMBOS = [(1, 1), (0, 0), (1, 2), (2, 1), (2, 2), (0, 1)]
