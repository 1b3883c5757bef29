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


def config3_spheres(dims=(508, 508, 508), seed=0, n=3):
    """The 508^3 configuration's emitters: ``n`` seeded spheres of radius 20-40 cells resting
    near the floor, away from the side walls."""
    rng = np.random.default_rng(seed)
    X, Y, Z = dims
    out = []
    for _ in range(n):
        r = float(rng.uniform(20.0, 40.0))
        out.append(dict(center=(float(rng.uniform(r + 8, X - r - 8)), r + 4.0, float(rng.uniform(r + 8, Z - r - 8))),
                        radius=r, fuel=1.0, temperature=1500.0))
    return out


def backward_divergence(flow, u):
    """computeDivergence (shaders.ts:344-364) in float32 with the kernel's operation order:
    (u - u[x-1]) mx + (v - v[y-1]) my + (w - w[z-1]) mz, clamped neighbours, metric =
    grid / max(domain, 0.001) from the uniform block ``u``. ``flow`` is (Z, Y, X, 4)."""
    f32 = np.float32
    m = [f32(u[k]) / max(f32(u[32 + k]), f32(0.001)) for k in range(3)]
    U, V, W = flow[..., 0], flow[..., 1], flow[..., 2]
    left = np.concatenate([U[:, :, :1], U[:, :, :-1]], axis=2)
    bottom = np.concatenate([V[:, :1], V[:, :-1]], axis=1)
    back = np.concatenate([W[:1], W[:-1]], axis=0)
    return ((U - left) * m[0] + (V - bottom) * m[1]) + (W - back) * m[2]
