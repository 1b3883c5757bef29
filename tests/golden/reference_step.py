"""The reference's own Fire-X step, executed on the CPU from its WGSL source text — TEST
INFRASTRUCTURE ONLY (fixture generation; it reads the reference tree, so it runs only where
that tree is present, never in the tests themselves).

The shaders are the reference's text, parsed and evaluated by tests/golden/wgsl_eval.py:
  * FIREX_COMPUTE_WGSL     src/sim/firex/shaders.ts:1-512 (initializeFields, simulate,
    computeDivergence, solvePressureGlobal, solvePressureTiled, projectVelocity, copyFlow);
  * FIREX_F16_PRESSURE_WGSL src/sim/firex/pressureShaders.ts:1-161 (solvePressureF16Tiled,
    projectVelocityF16);
  * FIREX_PARTICLE_WGSL    src/sim/firex/shaders.ts:514-825 (computeParticleDensity,
    integrateParticles, depositParticles), with sin / cos / tan / exp evaluated in double
    precision and rounded to f32 (hash11 scales one ULP of sin by 43758, so the droplets
    depend on which correctly-bounded sin is used: this is the choice the library and its
    oracle make).

The host side around them is restated here from src/sim/firex/FireXEngine.ts (the reference
host is TypeScript driving WebGPU, which cannot run on this machine):
  * buffers and bind groups of createResourceSet (:1536-1771): flow[2], species[2],
    pressure[2], correctionPressure[2], divergence, liquid, reaction, each bind group's
    nine bindings (computeGroup :1640-1663) and the f16 groups (:1723-1748);
  * reset / initializeFields (:843-852, :1933-1974): cleared buffers, the initialisation
    uniform (grid, oxygenRate, ambient 300 K) and the (groupsX, groupsY) dispatch;
  * writeUniforms (:2043-2113): the 44-float block from the engine parameters (defaults
    :422-451) and the 8-float f16 pressure block;
  * encodeSimulationStep (:2115-2276) with its three pressure branches, ping-pong indices,
    buffer clears and dispatch sizes; the step then advances simulationTime and frameIndex
    (renderOfflineFrameInternal :669-682);
  * the droplet state machine of encodeSimulationStep (:2158-2171: spray on -> initial
    droplets if parked, liquid cleared, density / integration / deposition over the
    particle bind group (:1772-1786), ping-pong; spray off -> liquid cleared and droplets
    parked) and writeParticleInitialState (:1976-2034, JavaScript doubles stored as f32).
Branch choice: the reference takes the heavy branches (B: f16 tiled, C: f32 tiled, cold
start) only from 64 Mi cells (:2175); `branch` forces one on a small grid so every branch's
kernels and bookkeeping run here.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

from tests.golden.wgsl_eval import Program, wgsl_from_ts

SHADERS = Path("src/sim/firex/shaders.ts")
PRESSURE_SHADERS = Path("src/sim/firex/pressureShaders.ts")

# FireXEngine.parameters defaults (FireXEngine.ts:422-451)
DEFAULT_PARAMETERS = dict(
    burnerSize=3.1, burnerDepth=2.7, sourceThickness=1.35, firePower=2.5, sourceLift=1.6, buoyancyScale=2.15,
    flamePersistence=1.45, airEntrainment=1.65, fuelRate=0.30, oxygenRate=1, heatEfficiency=0.86, vorticity=3.6,
    waterFlow=0, sprayAngle=10, waterEnabled=False, cameraYaw=-0.34, cameraPitch=0.03, cameraDistance=4.9,
    viewMode=0, aimHeight=0.42, nozzleType=0, exposure=1.25, frontDefinition=1.65, domainWidth=1.15,
    domainHeight=1.35, domainDepth=1.15, viewZoom=2.1, opticalDetailTarget=1024)


def load_programs(reference_root):
    root = Path(reference_root)
    src = (root / SHADERS).read_text()
    main = Program(wgsl_from_ts(src, "FIREX_COMPUTE_WGSL"))
    f16 = Program(wgsl_from_ts((root / PRESSURE_SHADERS).read_text(), "FIREX_F16_PRESSURE_WGSL"))
    particles = Program(wgsl_from_ts(src, "FIREX_PARTICLE_WGSL"), transcendentals="f64")
    return main, f16, particles


class ReferenceStep:
    """One Fire-X simulation run by the reference's kernels. Fields are numpy arrays in the
    reference's buffer layout (cell index x + X*(y + Y*z))."""

    def __init__(self, programs, dims, branch="A", P=8, R=8, parameters=None, cinematic=1, time_step=1 / 60,
                 particle_count=0):
        self.main, self.f16, self.sph = programs
        self.np = int(particle_count)
        self.particles = [np.zeros((self.np, 8), np.float32) for _ in range(2)]
        self.density = np.zeros((self.np, 4), np.float32)
        self.particle_index = 0
        self.particle_field_active = False
        self.liquid_may_contain_water = False
        self.X, self.Y, self.Z = dims
        self.N = self.X * self.Y * self.Z
        self.branch = branch
        self.P, self.R = P, R
        self.par = dict(DEFAULT_PARAMETERS, **(parameters or {}))
        self.cinematic = cinematic
        self.time_step = time_step
        self.half = branch == "B"
        ptype = np.float16 if self.half else np.float32
        N = self.N
        self.flow = [np.zeros((N, 4), np.float32) for _ in range(2)]
        self.species = [np.zeros((N, 4), np.float32) for _ in range(2)]
        self.pressure = [np.zeros(N, ptype) for _ in range(2)]
        # the heavy f32 fallback allocates 4-byte correction buffers (:1585-1594)
        self.correction = [np.zeros(1 if branch == "C" else N, ptype) for _ in range(2)]
        self.divergence = np.zeros(N, np.float32)
        self.liquid = np.zeros(N, np.uint32)
        self.reaction = np.zeros(N, np.float32)
        self.simulation_time = 0.0
        self.frame_index = 0
        self.species_index = 0
        self.pressure_index = 0
        self.reset()

    # ---- uniforms
    def uniforms(self, dt):
        """writeUniforms (FireXEngine.ts:2043-2113). Presentation-only slots (canvas size and
        aspect, ray steps, configuration.timeStep) do not enter the compute kernels; they
        hold 1, 1, 1, 0 and `time_step`."""
        p = self.par
        u = [self.X, self.Y, self.Z, self.N,
             dt, self.simulation_time, self.frame_index, self.time_step,
             p["fuelRate"], p["oxygenRate"], p["heatEfficiency"], p["vorticity"],
             p["waterFlow"], (p["sprayAngle"] * math.pi) / 180, 1 if p["waterEnabled"] else 0, 300,
             p["cameraYaw"], p["cameraPitch"], p["cameraDistance"], 1,
             1, 1, 0, self.np,
             p["viewMode"], p["aimHeight"], p["nozzleType"], p["exposure"],
             p["burnerSize"], p["burnerDepth"], p["sourceThickness"], p["firePower"],
             p["domainWidth"], p["domainHeight"], p["domainDepth"], 0,
             p["sourceLift"], p["buoyancyScale"], p["flamePersistence"], p["viewZoom"],
             p["airEntrainment"], p["frontDefinition"], 1 if self.cinematic else 0, p["opticalDetailTarget"]]
        return np.array(u, np.float64).astype(np.float32)  # Float32Array.set rounds each JS number

    def f16_uniforms(self):
        p = self.par
        return np.array([self.X, self.Y, self.Z, self.N, p["domainWidth"], p["domainHeight"], p["domainDepth"], 0],
                        np.float64).astype(np.float32)

    # ---- dispatch helpers
    def _group(self, flow_read, species_read, flow_write, species_write, pressure_read, pressure_write):
        """computeGroup (FireXEngine.ts:1640-1663): bindings 1-8 of the compute module."""
        return dict(flowIn=flow_read, speciesIn=species_read, flowOut=flow_write, speciesOut=species_write,
                    divergenceField=self.divergence, pressureIn=pressure_read, pressureOut=pressure_write,
                    liquidField=self.liquid)

    def _run(self, entry, group, workgroups=None, uniforms=None):
        prog = self.main
        for k, v in group.items():
            prog.bind(k, v)
        prog.bind_uniform("params", uniforms)
        if workgroups is None:
            workgroups = (math.ceil(self.X / 4), math.ceil(self.Y / 4), math.ceil(self.Z / 4))
        prog.run(entry, workgroups)

    def _run_f16(self, entry, pressure_read, pressure_write, flow_read, flow_write, workgroups=None):
        """createF16PressureGroup (FireXEngine.ts:1723-1740)."""
        prog = self.f16
        prog.bind("divergenceField", self.divergence)
        prog.bind("pressureIn", pressure_read)
        prog.bind("pressureOut", pressure_write)
        prog.bind("flowIn", flow_read)
        prog.bind("flowOut", flow_write)
        prog.bind_uniform("params", self.f16_uniforms())
        if workgroups is None:
            workgroups = (math.ceil(self.X / 4), math.ceil(self.Y / 4), math.ceil(self.Z / 4))
        prog.run(entry, workgroups)

    # ---- reset (FireXEngine.ts:843-852, initializeFields :1933-1974)
    def reset(self):
        self.simulation_time = 0.0
        self.frame_index = 0
        self.species_index = 0
        self.pressure_index = 0
        for bufs in (self.flow, self.species, self.pressure, self.correction):
            for b in bufs:
                b[...] = 0
        for b in (self.divergence, self.liquid, self.reaction):
            b[...] = 0
        u = np.zeros(44, np.float32)
        u[0:4] = [self.X, self.Y, self.Z, self.N]
        u[9] = self.par["oxygenRate"]
        u[15] = 300
        total = math.ceil(self.N / 256)
        gx = min(total, 65535)
        gy = math.ceil(total / gx)
        f, s, p = self.flow, self.species, self.pressure
        self._run("initializeFields", self._group(f[1], s[1], f[0], s[0], p[0], p[1]), (gx, gy, 1), u)
        self.particles = [np.zeros((self.np, 8), np.float32) for _ in range(2)]
        self.density = np.zeros((self.np, 4), np.float32)
        self.write_particle_initial_state(self.water_active())
        self.liquid_may_contain_water = False

    # ---- droplets
    def water_active(self):
        return bool(self.par["waterEnabled"]) and self.par["waterFlow"] > 0.001  # FireXEngine.ts:2537-2539

    def write_particle_initial_state(self, active):
        """writeParticleInitialState (FireXEngine.ts:1976-2034): JavaScript doubles, stored as
        f32 (Float32Array) at the end."""
        p = self.par
        out = np.zeros((self.np, 8), np.float64)
        aim_x = (0.52 - 0.035) * p["domainWidth"]
        aim_y = (p["aimHeight"] - 0.5) * p["domainHeight"]
        aim_len = math.hypot(aim_x, aim_y)
        base = (aim_x / aim_len, aim_y / aim_len, 0.0)
        tangent = (base[1], -base[0], 0.0)

        def hsh(v):
            h = math.sin(v * 12.9898 + 1.317) * 43758.5453
            return h - math.floor(h)

        spray = p["nozzleType"] >= 0.5
        for i in range(self.np):
            phase = i / self.np
            angle = hsh(i * 3.771 + 4.91) * math.pi * 2
            radial = math.sqrt(hsh(i * 3.771 + 0.17))
            cone = math.tan((p["sprayAngle"] * math.pi) / 180) * radial * (0.72 if spray else 0.1)
            disk_x, disk_y, disk_z = tangent[0] * math.cos(angle), tangent[1] * math.cos(angle), -math.sin(angle)
            dx, dy, dz = base[0] + disk_x * cone, base[1] + disk_y * cone, disk_z * cone
            dl = math.hypot(dx, dy, dz)
            dx, dy, dz = dx / dl, dy / dl, dz / dl
            var = 0.24 if spray else 0.05
            speed = (0.82 + p["waterFlow"] * 0.82) * (1 - var * 0.5 + hsh(i * 3.771 + 9.37) * var)
            age = phase * 0.72
            origin_r = 0.006 if spray else 0.0028
            out[i, 0] = 0.035 + (disk_x * radial * origin_r + dx * speed * age) / p["domainWidth"]
            out[i, 1] = max(0.012, 0.5 + (disk_y * radial * origin_r + dy * speed * age - 0.29 * age * age)
                            / p["domainHeight"])
            out[i, 2] = 0.5 + (disk_z * radial * origin_r + dz * speed * age) / p["domainDepth"]
            out[i, 3] = age if active else -phase * 0.72
            if active:
                out[i, 4:8] = (dx * speed, dy * speed - 0.58 * age, dz * speed, 0.52 + p["waterFlow"] * 0.88)
        init = out.astype(np.float32)
        self.particles = [init.copy(), init.copy()]
        self.particle_index = 0
        self.particle_field_active = active

    def _particle_pass(self, u):
        """FireXEngine.ts:2158-2171 and the particle bind groups (:1772-1786)."""
        if self.water_active():
            if not self.particle_field_active:
                self.write_particle_initial_state(True)
            self.liquid[...] = 0
            i = self.particle_index
            prog = self.sph
            prog.bind("flowField", self.flow[0])
            prog.bind("particlesIn", self.particles[i])
            prog.bind("particlesOut", self.particles[1 - i])
            prog.bind("densityData", self.density)
            prog.bind("liquidField", self.liquid)
            prog.bind_uniform("params", u)
            groups = (math.ceil(self.np / 64), 1, 1)
            for entry in ("computeParticleDensity", "integrateParticles", "depositParticles"):
                prog.run(entry, groups)
            self.particle_index = 1 - i
            self.liquid_may_contain_water = True
        elif self.liquid_may_contain_water or self.particle_field_active:
            self.liquid[...] = 0
            self.write_particle_initial_state(False)
            self.liquid_may_contain_water = False

    # ---- encodeSimulationStep (FireXEngine.ts:2115-2276) and the counters (:669-682)
    def step(self, dt, trace=None):
        """One step. `trace`, when a dict, receives copies of the buffers after each pass."""
        u = self.uniforms(dt)
        f, s, p, c = self.flow, self.species, self.pressure, self.correction
        X, Y, Z = self.X, self.Y, self.Z
        rec = (lambda name, arr: trace.__setitem__(name, arr.copy())) if trace is not None else (lambda *a: None)
        if self.np > 0:
            self._particle_pass(u)
        si = self.species_index
        sim_group = (self._group(f[0], s[0], f[1], s[1], p[0], self.reaction) if si == 0 else
                     self._group(f[0], s[1], f[1], s[0], p[0], self.reaction))
        self._run("simulate", sim_group, uniforms=u)
        self.species_index = 1 - si
        rec("simulate.flow", f[1])
        rec("simulate.species", s[1 - si])
        rec("simulate.reaction", self.reaction)
        self._run("computeDivergence", self._group(f[1], s[0], f[0], s[1], p[0], p[1]), uniforms=u)
        rec("divergence", self.divergence)
        heavy_dispatch = (math.ceil(X / 8), math.ceil(Y / 8), math.ceil(Z / 4))
        if self.branch == "B":
            for _ in range(self.P):
                pi = self.pressure_index
                self._run_f16("solvePressureF16Tiled", p[pi], p[1 - pi], f[1], f[0], heavy_dispatch)
                self.pressure_index = 1 - pi
            rec("primary.pressure", p[self.pressure_index])
            pi = self.pressure_index
            self._run_f16("projectVelocityF16", p[pi], p[1 - pi], f[1], f[0])
            rec("primary.flow", f[0])
            self._run("computeDivergence", self._group(f[0], s[0], f[1], s[1], p[0], p[1]), uniforms=u)
            rec("residual.divergence", self.divergence)
            c[0][...] = 0
            c[1][...] = 0
            ci = 0
            for _ in range(self.R):
                self._run_f16("solvePressureF16Tiled", c[ci], c[1 - ci], f[0], f[1], heavy_dispatch)
                ci = 1 - ci
            rec("residual.pressure", c[ci])
            self._run_f16("projectVelocityF16", c[ci], c[1 - ci], f[0], f[1])
        elif self.branch == "C":
            p[0][...] = 0
            p[1][...] = 0
            self.pressure_index = 0
            for _ in range(self.P):
                pi = self.pressure_index
                self._run("solvePressureTiled", self._group(f[0], s[0], f[1], s[1], p[pi], p[1 - pi]), heavy_dispatch, u)
                self.pressure_index = 1 - pi
            rec("primary.pressure", p[self.pressure_index])
            pi = self.pressure_index
            self._run("projectVelocity", self._group(f[1], s[0], f[0], s[1], p[pi], p[1 - pi]), uniforms=u)
            rec("primary.flow", f[0])
            self._run("computeDivergence", self._group(f[0], s[0], f[1], s[1], p[0], p[1]), uniforms=u)
            rec("residual.divergence", self.divergence)
            p[0][...] = 0
            p[1][...] = 0
            ci = 0
            for _ in range(self.R):
                self._run("solvePressureTiled", self._group(f[0], s[0], f[1], s[1], p[ci], p[1 - ci]), heavy_dispatch, u)
                ci = 1 - ci
            rec("residual.pressure", p[ci])
            self._run("projectVelocity", self._group(f[0], s[0], f[1], s[1], p[ci], c[0]), uniforms=u)
        else:
            for _ in range(self.P):
                pi = self.pressure_index
                self._run("solvePressureGlobal", self._group(f[0], s[0], f[1], s[1], p[pi], p[1 - pi]), uniforms=u)
                self.pressure_index = 1 - pi
            rec("primary.pressure", p[self.pressure_index])
            pi = self.pressure_index
            self._run("projectVelocity", self._group(f[1], s[0], f[0], s[1], p[pi], p[1 - pi]), uniforms=u)
            rec("primary.flow", f[0])
            self._run("computeDivergence", self._group(f[0], s[0], f[1], s[1], p[0], p[1]), uniforms=u)
            rec("residual.divergence", self.divergence)
            c[0][...] = 0
            c[1][...] = 0
            ci = 0
            for _ in range(self.R):
                self._run("solvePressureGlobal", self._group(f[0], s[0], f[1], s[1], c[ci], c[1 - ci]), uniforms=u)
                ci = 1 - ci
            rec("residual.pressure", c[ci])
            self._run("projectVelocity", self._group(f[0], s[0], f[1], s[1], c[ci], p[0]), uniforms=u)
        rec("residual.flow", f[1])
        self._run("copyFlow", self._group(f[1], s[0], f[0], s[1], p[0], c[0]), uniforms=u)
        self.simulation_time += dt
        self.frame_index += 1

    # ---- the resident state, in the order of the library's field ids
    def current(self):
        out = dict(flow=self.flow[0].copy(), species=self.species[self.species_index].copy(),
                   pressure=self.pressure[self.pressure_index].astype(np.float32),
                   divergence=self.divergence.copy(), reaction=self.reaction.copy(), liquid=self.liquid.copy())
        if self.np > 0:
            out["particles"] = self.particles[self.particle_index].copy()
        return out
