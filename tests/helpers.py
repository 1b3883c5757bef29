"""Scene builders and comparison helpers shared by the parity tests."""
from __future__ import annotations

import numpy as np

from fire_b200.sim import make_options

DT = 1.0 / 60.0


def sphere_options(dims, P=8, R=8, *, seed=7, noise=0.05, jitter=0.1, spheres=None, **kw):
    """Config-1-style sphere scene scaled to ``dims``: one sphere near the floor."""
    X, Y, Z = dims
    if spheres is None:
        r = max(2.0, min(X, Z) / 8.0)
        spheres = [dict(center=(X / 2, Y / 12 + r / 2, Z / 2), radius=r, fuel=1.0, temperature=1500.0)]
    return make_options(pressure_iterations=P, correction_iterations=R, seed=seed, velocity_noise=noise,
                        emission_jitter=jitter, spheres=spheres, **kw)


def burner_options(P=8, R=8, **kw):
    return make_options(pressure_iterations=P, correction_iterations=R, **kw)


def copy_state(src, dst, fields=("flow", "species", "pressure", "liquid")):
    """Makes dst hold src's resident state and counters."""
    st = src.state
    dst.set_state(st["simulation_time"], st["frame_index"], st["species_index"], st["pressure_index"])
    for f in fields:
        dst.write(f, src.read(f))


def max_abs(a, b) -> float:
    return float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64)))) if a.size else 0.0


def rel_l2(a, b, ref=None) -> float:
    """||a - b||_2 / ||ref||_2 (ref defaults to b)."""
    ref = b if ref is None else ref
    den = float(np.linalg.norm(ref.astype(np.float64).ravel()))
    return float(np.linalg.norm((a.astype(np.float64) - b.astype(np.float64)).ravel())) / max(den, 1e-300)


def interior(a):
    """Interior cells (one-cell outer shell excluded), arrays shaped (Z, Y, X, ...)."""
    return a[1:-1, 1:-1, 1:-1]
