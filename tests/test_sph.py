"""SPH droplets and liquid deposition (FIREX_PARTICLE_WGSL, shaders.ts:514-825; the particle
state machine of FireXEngine.ts:2158-2171 and writeParticleInitialState, :1976-2034).

CPU: the oracle's droplet pass is pinned against a scalar numpy restatement written from
the WGSL (one step from a mid-spray state, spray and jet nozzles, bit for bit), its initial
state against a restatement of the host code, and its state machine (water off: no
droplets, empty liquid; on: droplets spawn; off again: liquid cleared, droplets parked).
GPU: from the oracle's state the CUDA pass gives the same droplets and the same liquid
field bit for bit; the engine follows the same state machine; a batch whose members spray
or not equals each member alone; ten steps from reset stay close to the oracle's."""
from __future__ import annotations

import math

import numpy as np
import pytest

from fire_b200.sim import FireXBatch, FireXSim
from oracle.oracle import OracleSim
from tests.helpers import DT, copy_state, max_abs, sphere_options

F = np.float32
WATER = {"waterEnabled": True, "waterFlow": 0.8, "sprayAngle": 25}


def _start(sim, nozzle, **extra):
    for k, v in {**WATER, "nozzleType": nozzle, **extra}.items():
        sim.set_parameter(k, v)
    sim.reset()
    return sim


# ---- numpy restatement of the WGSL, float32 scalar by scalar ---------------------------
def _sin(x):
    return F(math.sin(float(x)))


def _fract(x):
    return F(x - F(math.floor(float(x))))


def _hash11(v):
    return _fract(_sin(F(v) * F(12.9898) + F(1.317)) * F(43758.5453))


def _len(v):
    return F(np.sqrt(F(F(v[0] * v[0]) + F(v[1] * v[1])) + F(v[2] * v[2])))


def _max(a, b):
    return b if a < b else a


def _clamp(x, lo, hi):
    x = _max(F(x), F(lo))
    return F(hi) if F(hi) < x else x


def _norm(v):
    n = _len(v)
    return np.array([v[0] / n, v[1] / n, v[2] / n], dtype=F)


def _cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], dtype=F)


class Wgsl:
    """computeParticleDensity, integrateParticles, depositParticles for one step."""

    def __init__(self, u, dims):
        self.u = np.asarray(u, dtype=F)
        self.X, self.Y, self.Z = dims
        self.ext = np.array([_max(self.u[32 + i], F(0.001)) for i in range(3)], dtype=F)
        self.spray = self.u[26] >= F(0.5)
        self.radius = F(0.060) if self.spray else F(0.038)

    def cell(self, x, y, z):
        x, y, z = min(max(x, 0), self.X - 1), min(max(y, 0), self.Y - 1), min(max(z, 0), self.Z - 1)
        return x + self.X * (y + self.Y * z)

    def density(self, p):
        out = np.zeros((len(p), 4), dtype=F)
        for i in range(len(p)):
            if p[i, 1, 3] <= F(0.0001):
                continue
            de, near = F(0), F(0)
            for j in range(len(p)):
                if j == i or p[j, 1, 3] <= F(0.0001):
                    continue
                d = _len((p[i, 0, :3] - p[j, 0, :3]) * self.ext)
                if F(0.00001) < d < self.radius:
                    q = F(F(1) - d / self.radius)
                    de = F(de + q * q)
                    near = F(near + F(q * q) * q)
            rest = F(F(2.7) + self.u[12] * F(0.9))
            out[i] = [de, near, F(_max(F(de - rest), F(0)) * F(0.055)), F(near * F(0.065))]
        return out

    def direction(self):
        target = np.array([0.52, _clamp(self.u[25], 0.08, 0.82), 0.5], dtype=F)
        return _norm((target - np.array([0.035, 0.5, 0.5], dtype=F)) * self.ext)

    def spawn(self, i, cycle):
        u = self.u
        seed = F(F(i) * F(3.771) + F(cycle) * F(19.173))
        radial = F(np.sqrt(_hash11(seed + F(0.17))))
        angular = F(_hash11(seed + F(4.91)) * F(6.2831853))
        speed_r = _hash11(seed + F(9.37))
        d = self.direction()
        tangent = _norm(_cross(d, np.array([0, 0, 1], dtype=F)))
        bitangent = _norm(_cross(d, tangent))
        disk = tangent * F(math.cos(float(angular))) + bitangent * _sin(angular)
        cone = F(F(F(math.tan(float(_clamp(u[13], 0.005, 0.78)))) * radial) * (F(0.72) if self.spray else F(0.10)))
        launch = _norm(d + disk * cone)
        radius = F(0.006) if self.spray else F(0.0028)
        origin = np.array([0.035, 0.5, 0.5], dtype=F) + ((disk * radial) * radius) / self.ext
        sv = F(0.24) if self.spray else F(0.05)
        lo, hi = F(F(1) - sv * F(0.5)), F(F(1) + sv * F(0.5))
        speed = F(F(F(0.82) + u[12] * F(0.82)) * F(F(lo * F(F(1) - speed_r)) + F(hi * speed_r)))
        return np.array([[*origin, 0.0], [*(launch * speed), F(0.52) + u[12] * F(0.88)]], dtype=F)

    def integrate(self, p, dens, flow):
        u, dt = self.u, self.u[4]
        water_on = u[14] >= F(0.5) and u[12] > F(0.001)
        out = p.copy()
        for i in range(len(p)):
            if dt <= F(0):
                continue
            if p[i, 1, 3] <= F(0.0001):
                wait = F(p[i, 0, 3] + dt)
                if water_on and wait >= F(0):
                    out[i] = self.spawn(i, F(wait + u[6]))
                else:
                    out[i] = [[0.035, 0.5, 0.5, F(-0.72) if wait > F(0) else wait], [0, 0, 0, 0]]
                continue
            lifetime = F(F(0.88) + _hash11(F(F(i) * F(2.31) + F(7.0))) * F(0.52))
            next_age = F(p[i, 0, 3] + dt)
            pos, vel = p[i, 0, :3].copy(), p[i, 1, :3].copy()
            if next_age >= lifetime or (pos < F(-0.03)).any() or (pos > F(1.03)).any():
                if water_on:
                    out[i] = self.spawn(i, F(next_age + u[6]))
                else:
                    out[i] = [[0.035, 0.5, 0.5, -_hash11(F(F(i) * F(8.17))) * F(0.72)], [0, 0, 0, 0]]
                continue
            pa, va = np.zeros(3, F), np.zeros(3, F)
            for j in range(len(p)):
                if j == i or p[j, 1, 3] <= F(0.0001):
                    continue
                sep = (pos - p[j, 0, :3]) * self.ext
                d = _len(sep)
                if F(0.00001) < d < self.radius:
                    q = F(F(1) - d / self.radius)
                    direction = sep / d
                    pr = F(F(dens[i, 2] + dens[j, 2]) * q)
                    npr = F(F(F(dens[i, 3] + dens[j, 3]) * q) * q)
                    pa = pa + direction * F(pr + npr)
                    va = va + (p[j, 1, :3] - vel) * F(q * F(0.018))
            g = flow[self.cell(*(int(_clamp(pos[k], 0, 0.99999) * u[k]) for k in range(3)))]
            t = _clamp(F(g[3] - F(380)) / F(F(1500) - F(380)), 0, 1)
            heat = F(F(t * t) * F(F(3) - F(2) * t))
            acc = np.array([0, -0.58, 0], dtype=F) + (g[:3] - vel) * F(F(0.30) + heat * F(0.18))
            acc = acc + (pa * (F(1) if self.spray else F(0.055)) + va * (F(1) if self.spray else F(2.2)))
            vel = vel + acc * dt
            nxt = pos + (vel * dt) / self.ext
            if nxt[1] < F(0.012):
                nxt[1] = F(0.012)
                vel[1] = F(abs(vel[1]) * F(0.18))
                vel[0], vel[2] = vel[0] * F(0.72), vel[2] * F(0.72)
            for k in (0, 2):
                if nxt[k] < F(0.008) or nxt[k] > F(0.992):
                    nxt[k] = _clamp(nxt[k], 0.008, 0.992)
                    vel[k] = vel[k] * F(-0.24)
            mass = F(p[i, 1, 3] * F(math.exp(float(F(F(-heat * dt) * F(0.34))))))
            out[i] = [[*nxt, next_age], [*(_clamp(v, -2, 2) for v in vel), mass]]
        return out

    def corner(self, liq, c, w, m):
        liq[self.cell(*c)] += np.uint32(int(_clamp(F(F(w * m) * F(4096)), 0, 65535)))

    def deposit_at(self, liq, pos, mass):
        vp = pos * self.u[:3] - F(0.5)
        if not self.spray:
            b = [int(math.floor(float(v))) for v in vp]
            f = np.array([_fract(v) for v in vp], dtype=F)
            iv = F(1) - f
            m = F(mass * F(0.20))
            for dz in (0, 1):
                for dy in (0, 1):
                    for dx in (0, 1):
                        w = F(F((f[0] if dx else iv[0]) * (f[1] if dy else iv[1])) * (f[2] if dz else iv[2]))
                        self.corner(liq, (b[0] + dx, b[1] + dy, b[2] + dz), w, m)
            return
        c = [int(np.rint(v)) for v in vp]  # round half to even, as WGSL round()
        ks = []
        for oz in (-1, 0, 1):
            for oy in (-1, 0, 1):
                for ox in (-1, 0, 1):
                    d = _len(vp - np.array([c[0] + ox, c[1] + oy, c[2] + oz], dtype=F))
                    ks.append(((c[0] + ox, c[1] + oy, c[2] + oz), _max(F(0), F(F(1) - d * F(0.52)))))
        total = F(0)
        for _, k in ks:
            total = F(total + k * k)
        for cell, k in ks:
            self.corner(liq, cell, F(F(k * k) / _max(total, F(0.0001))), mass)

    def deposit(self, pin, pout, liq):
        for i in range(len(pout)):
            pos, mass = pout[i, 0, :3], pout[i, 1, 3]
            if mass <= F(0.0001) or (pos < F(0)).any() or (pos >= F(1)).any():
                continue
            disp = pos - pin[i, 0, :3]
            if not (pin[i, 1, 3] > F(0.0001) and pout[i, 0, 3] >= pin[i, 0, 3] and _len(disp * self.ext) < F(0.20)):
                self.deposit_at(liq, pos, mass)
                continue
            for k in range(3):
                self.deposit_at(liq, pin[i, 0, :3] + disp * (F(k) / F(2)), F(mass / F(3)))


def _initial_state(params, dims_m, n, active):
    """writeParticleInitialState in double, stored as float32."""
    w, h, d = dims_m
    ax, ay = (0.52 - 0.035) * w, (params["aimHeight"] - 0.5) * h
    al = math.hypot(ax, ay)
    base, tangent = (ax / al, ay / al, 0.0), (ay / al, -ax / al, 0.0)
    hsh = lambda v: (lambda x: x - math.floor(x))(math.sin(v * 12.9898 + 1.317) * 43758.5453)
    spray = params["nozzleType"] >= 0.5
    out = np.zeros((n, 2, 4), dtype=F)
    for i in range(n):
        phase = i / n
        angle = hsh(i * 3.771 + 4.91) * math.pi * 2
        radial = math.sqrt(hsh(i * 3.771 + 0.17))
        cone = math.tan(params["sprayAngle"] * math.pi / 180) * radial * (0.72 if spray else 0.1)
        dx_, dy_, dz_ = tangent[0] * math.cos(angle), tangent[1] * math.cos(angle), -math.sin(angle)
        v = [base[0] + dx_ * cone, base[1] + dy_ * cone, dz_ * cone]
        ln = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
        v = [c / ln for c in v]
        sv = 0.24 if spray else 0.05
        speed = (0.82 + params["waterFlow"] * 0.82) * (1 - sv * 0.5 + hsh(i * 3.771 + 9.37) * sv)
        age = phase * 0.72
        r0 = 0.006 if spray else 0.0028
        out[i, 0] = [0.035 + (dx_ * radial * r0 + v[0] * speed * age) / w,
                     max(0.012, 0.5 + (dy_ * radial * r0 + v[1] * speed * age - 0.29 * age * age) / h),
                     0.5 + (dz_ * radial * r0 + v[2] * speed * age) / d, age if active else -phase * 0.72]
        if active:
            out[i, 1] = [v[0] * speed, v[1] * speed - 0.58 * age, v[2] * speed, 0.52 + params["waterFlow"] * 0.88]
    return out


def _params(sim):
    names = ("aimHeight", "nozzleType", "sprayAngle", "waterFlow", "domainWidth", "domainHeight", "domainDepth")
    return {k: sim.get_parameter(k) for k in names}


# ---- CPU: the oracle against the restatements ------------------------------------------
@pytest.mark.parametrize("nozzle", [0, 1])
@pytest.mark.parametrize("active", [False, True])
def test_oracle_initial_state_matches_host_restatement(nozzle, active):
    dims = (16, 24, 16)
    o = OracleSim(dims, sphere_options(dims, P=4, R=4, particle_count=96))
    if active:
        _start(o, nozzle)
    else:
        o.set_parameter("nozzleType", nozzle)
        o.reset()
    prm = _params(o)
    ref = _initial_state(prm, (prm["domainWidth"], prm["domainHeight"], prm["domainDepth"]), 96, active)
    assert np.array_equal(o.read_particles(), ref)


@pytest.mark.parametrize("nozzle", [0, 1])
def test_oracle_droplet_pass_matches_wgsl_restatement(nozzle):
    """One step from a mid-spray state: droplets and liquid bit for bit."""
    dims = (16, 24, 16)
    o = OracleSim(dims, sphere_options(dims, P=4, R=4, particle_count=96))
    _start(o, nozzle)
    o.step(6, DT)
    pin, flow, u = o.read_particles(), o.read("flow").reshape(-1, 4), o.uniforms(DT)
    w = Wgsl(u, dims)
    dens = w.density(pin)
    assert (dens[:, 0] > 0).sum() > 10  # droplets do interact
    pout = w.integrate(pin, dens, flow)
    liq = np.zeros(np.prod(dims), dtype=np.uint32)
    w.deposit(pin, pout, liq)
    o.step(1, DT)
    got = o.read_particles()
    assert np.array_equal(got, pout), float(np.abs(got - pout).max())
    assert np.array_equal(o.read("liquid").reshape(-1), liq)
    assert liq.sum() > 0


def test_oracle_water_state_machine():
    dims = (16, 24, 16)
    o = OracleSim(dims, sphere_options(dims, P=4, R=4, particle_count=64))
    o.step(2, DT)  # water off: droplets parked, nothing deposited
    p = o.read_particles()
    assert (p[:, 1] == 0).all() and (p[:, 0, 3] <= 0).all()
    assert not o.read("liquid").any()
    for k, v in {**WATER, "nozzleType": 1}.items():
        o.set_parameter(k, v)
    o.step(3, DT)  # turned on mid-run: the active initial state is written, then stepped
    assert (o.read_particles()[:, 1, 3] > 0).any() and o.read("liquid").any()
    o.set_parameter("waterEnabled", False)
    o.step(1, DT)  # off again: liquid cleared, droplets back to the parked initial state
    assert not o.read("liquid").any()
    prm = _params(o)
    ref = _initial_state(prm, (prm["domainWidth"], prm["domainHeight"], prm["domainDepth"]), 64, False)
    assert np.array_equal(o.read_particles(), ref)


def test_oracle_zero_particles_and_size_checks():
    dims = (8, 12, 8)
    o = OracleSim(dims, sphere_options(dims, P=2, R=2, particle_count=0))
    _start(o, 1)
    o.step(2, DT)
    assert o.read_particles().shape == (0, 2, 4)
    assert not o.read("liquid").any()


# ---- GPU: the CUDA pass against the oracle -----------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("nozzle", [0, 1])
@pytest.mark.parametrize("dims,n", [((16, 24, 16), 96), ((64, 96, 64), 640), ((48, 64, 40), 1537)])
def test_gpu_droplet_step_bit_exact(dims, n, nozzle):
    opts = lambda: sphere_options(dims, P=8, R=8, particle_count=n)
    o = _start(OracleSim(dims, opts()), nozzle)
    o.step(5, DT)
    g = _start(FireXSim(dims, opts()), nozzle)
    copy_state(o, g)
    g.write_particles(o.read_particles())
    o.step(1, DT)
    g.step(1, DT)
    po, pg = o.read_particles(), g.read_particles()
    assert np.array_equal(pg, po), (int((pg != po).sum()), float(np.abs(pg - po).max()))
    lo, lg = o.read("liquid"), g.read("liquid")
    assert lo.any() and np.array_equal(lg, lo), int((lg != lo).sum())


@pytest.mark.gpu
def test_gpu_water_state_machine_matches_oracle():
    dims = (32, 48, 32)
    opts = lambda: sphere_options(dims, P=6, R=6, particle_count=256)
    o, g = OracleSim(dims, opts()), FireXSim(dims, opts())
    for s in (o, g):
        s.step(2, DT)
    assert np.array_equal(g.read_particles(), o.read_particles())
    dry = g.diagnostics["launches_per_step"]
    for s in (o, g):
        for k, v in {**WATER, "nozzleType": 1}.items():
            s.set_parameter(k, v)
        s.step(1, DT)
    assert g.diagnostics["launches_per_step"] == dry + 2  # liquid clear + density, integrate + deposit
    # the first step with water on starts from states that agree within the step's float
    # tolerance, and the droplets read only their nearest cell of the flow
    assert max_abs(g.read_particles(), o.read_particles()) <= 1e-4
    for s in (o, g):
        s.set_parameter("waterEnabled", False)
        s.step(1, DT)
    assert not g.read("liquid").any()
    assert np.array_equal(g.read_particles(), o.read_particles())


@pytest.mark.gpu
def test_gpu_batch_with_and_without_water_equals_alone():
    cases = [((32, 48, 32), 256, 1), ((16, 24, 16), 0, 1), ((48, 64, 40), 640, None), ((32, 40, 24), 384, 0)]

    def make(dims, n, nozzle, i):
        s = FireXSim(dims, sphere_options(dims, P=6, R=6, seed=5 + i, particle_count=n))
        return _start(s, nozzle) if nozzle is not None else s

    alone = []
    for i, (d, n, nz) in enumerate(cases):
        s = make(d, n, nz, i)
        s.step(4, DT)
        alone.append(s)
    b = FireXBatch()
    members = [make(d, n, nz, i) for i, (d, n, nz) in enumerate(cases)]
    for m in members:
        b.add(m)
    b.step(4, DT)
    b.sync()
    for m, s in zip(members, alone):
        assert np.array_equal(m.read_particles(), s.read_particles())
        for f in ("flow", "species", "pressure", "liquid", "reaction"):
            assert np.array_equal(m.read(f), s.read(f)), f


@pytest.mark.gpu
def test_gpu_droplet_trajectory_tracks_oracle():
    dims = (64, 96, 64)
    opts = lambda: sphere_options(dims, P=16, R=16, particle_count=640)
    o, g = _start(OracleSim(dims, opts()), 1), _start(FireXSim(dims, opts()), 1)
    for s in (o, g):
        s.step(10, DT)
    po, pg = o.read_particles(), g.read_particles()
    same = np.all(po == pg, axis=(1, 2))
    assert same.mean() >= 0.9, same.mean()
    lo, lg = o.read("liquid").astype(np.float64), g.read("liquid").astype(np.float64)
    assert abs(lg.sum() - lo.sum()) <= 0.02 * lo.sum()
