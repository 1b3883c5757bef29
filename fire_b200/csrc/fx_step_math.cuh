// fx_step_math.cuh — per-cell math of the Fire-X step, written once and instantiated
// by every kernel variant (f32 storage, mixed storage, batched).
//
// Each function states the reference lines it computes. Storage is abstracted by an
// accessor (Acc) so that the same arithmetic serves all layouts:
//   float4 Acc::flow(long long i)        velocity (u v w) and temperature T
//   float4 Acc::species(long long i)     fuel, O2, products, vapor
//   uint32_t Acc::liquid(long long i)    deposited liquid, fixed point x4096
#pragma once

#include "fx_device.cuh"

// trilinearFlow / trilinearSpecies (shaders.ts:61-95): 8-tap trilinear sample at
// position - 0.5, clamped to [0, dims - 1.001]; taps use clamped addressing.
template <class Load>
FXD float4 fx_trilinear(const FxGrid& g, const float* u, float px, float py, float pz, Load load) {
    float sx = fx_clamp(px - 0.5f, 0.0f, u[U_GRID_X] - FC(1.001));
    float sy = fx_clamp(py - 0.5f, 0.0f, u[U_GRID_Y] - FC(1.001));
    float sz = fx_clamp(pz - 0.5f, 0.0f, u[U_GRID_Z] - FC(1.001));
    float flx = floorf(sx), fly = floorf(sy), flz = floorf(sz);
    int bx = (int)flx, by = (int)fly, bz = (int)flz;
    float fx = sx - flx, fy = sy - fly, fz = sz - flz;
    float4 c000 = load(g.idx(bx, by, bz)), c100 = load(g.idx(bx + 1, by, bz));
    float4 c010 = load(g.idx(bx, by + 1, bz)), c110 = load(g.idx(bx + 1, by + 1, bz));
    float4 c001 = load(g.idx(bx, by, bz + 1)), c101 = load(g.idx(bx + 1, by, bz + 1));
    float4 c011 = load(g.idx(bx, by + 1, bz + 1)), c111 = load(g.idx(bx + 1, by + 1, bz + 1));
    float4 z0 = fx_mix4(fx_mix4(c000, c100, fx), fx_mix4(c010, c110, fx), fy);
    float4 z1 = fx_mix4(fx_mix4(c001, c101, fx), fx_mix4(c011, c111, fx), fy);
    return fx_mix4(z0, z1, fz);
}

// emitter (shaders.ts:101-133): analytic elliptical-Gaussian burner with cellular,
// lobe and pulse texture, at normalised position (nx, ny, nz).
FXD float fx_burner(const float* u, float nx, float ny, float nz) {
    float time = u[U_TIME];
    float3 ext = fx_extent(u);
    float px = nx * ext.x, py = ny * ext.y, pz = nz * ext.z;
    float cx = ext.x * 0.5f + sinf(time * FC(1.73)) * FC(0.013);
    float cy = FC(0.075);
    float cz = ext.z * 0.5f + cosf(time * FC(1.37)) * FC(0.011);
    float ox = px - cx, oy = py - cy, oz = pz - cz;
    const float baseRadius = FC(0.1422673539502299);  // sqrt(0.02024), a WGSL const-expression
    float radiusX = fx_min(baseRadius * fx_clamp(u[U_BURNER_X], FC(0.35), FC(3.2)), ext.x * FC(0.42));
    float radiusZ = fx_min(baseRadius * fx_clamp(u[U_BURNER_Z], FC(0.35), FC(3.2)), ext.z * FC(0.42));
    float thickness = fx_clamp(u[U_THICKNESS], FC(0.35), FC(2.5));
    float radial = ox * ox / (radiusX * radiusX) + oz * oz / (radiusZ * radiusZ);
    float vertical = oy * oy / (FC(0.0022) * thickness * thickness);
    float cellular = FC(0.76) + FC(0.24) * sinf(px * 49.0f + time * FC(5.2)) * sinf(pz * 43.0f - time * FC(4.4));
    float lobeArg = sinf(ox / fx_max(radiusX, FC(0.001)) * FC(6.2) + time * FC(1.7)) *
                    sinf(oz / fx_max(radiusZ, FC(0.001)) * FC(5.4) - time * FC(1.3));
    float lobes = fx_mix(FC(0.48), FC(1.18), fx_smoothstep(FC(-0.42), FC(0.48), lobeArg));
    float texture = fx_mix(cellular, cellular * lobes, fx_clamp(u[U_CINEMATIC], 0.0f, 1.0f));
    float pulse = FC(0.84) + FC(0.16) * sinf(time * FC(3.7) + px * 27.0f + pz * 21.0f);
    return expf(-(radial + vertical)) * texture * pulse;
}

struct FxCellOut {
    float4 flow;
    float4 species;
    float reaction;
};

// simulate (shaders.ts:151-342) for cell (x, y, z): advection, diffusion, source,
// boundary ambient, liquid cooling, entrainment, Arrhenius burn, vorticity confinement,
// turbulence, buoyancy, spray momentum, radiation, open-top outflow and wall clamps.
template <class Acc>
FXD FxCellOut fx_simulate_cell(const FxParams& P, const FxGrid& g, int x, int y, int z, const Acc& a) {
    const float* u = P.u;
    const int X = g.X, Y = g.Y, Z = g.Z;
    long long id = g.idx(x, y, z);
    float picx = (float)x + 0.5f, picy = (float)y + 0.5f, picz = (float)z + 0.5f;
    float nx = picx / u[U_GRID_X], ny = picy / u[U_GRID_Y], nz = picz / u[U_GRID_Z];
    float dt = u[U_DT];

    float4 orig = a.flow(id);
    float3 metric = fx_metric(u);
    float btx = picx - orig.x * dt * metric.x;
    float bty = picy - orig.y * dt * metric.y;
    float btz = picz - orig.z * dt * metric.z;
    float4 flow = fx_trilinear(g, u, btx, bty, btz, [&](long long i) { return a.flow(i); });
    float4 species = fx_trilinear(g, u, btx, bty, btz, [&](long long i) { return a.species(i); });
    species = make_float4(fx_max(species.x, 0.0f), fx_max(species.y, 0.0f), fx_max(species.z, 0.0f),
                          fx_max(species.w, 0.0f));

    float4 left = a.flow(g.idx(x - 1, y, z)), right = a.flow(g.idx(x + 1, y, z));
    float4 bottom = a.flow(g.idx(x, y - 1, z)), top = a.flow(g.idx(x, y + 1, z));
    float4 back = a.flow(g.idx(x, y, z - 1)), front = a.flow(g.idx(x, y, z + 1));

    {  // 6-neighbour diffusion of velocity and temperature (shaders.ts:177-180)
        float vax = (left.x + right.x + bottom.x + top.x + back.x + front.x) / 6.0f;
        float vay = (left.y + right.y + bottom.y + top.y + back.y + front.y) / 6.0f;
        float vaz = (left.z + right.z + bottom.z + top.z + back.z + front.z) / 6.0f;
        float vm = fx_clamp(dt * FC(0.32), 0.0f, FC(0.12));
        flow.x = fx_mix(flow.x, vax, vm);
        flow.y = fx_mix(flow.y, vay, vm);
        flow.z = fx_mix(flow.z, vaz, vm);
        float ta = (left.w + right.w + bottom.w + top.w + back.w + front.w) / 6.0f;
        flow.w = fx_mix(flow.w, ta, fx_clamp(dt * FC(0.18), 0.0f, FC(0.08)));
    }
    {  // species diffusion (shaders.ts:182-187)
        float4 sl = a.species(g.idx(x - 1, y, z)), sr = a.species(g.idx(x + 1, y, z));
        float4 sb = a.species(g.idx(x, y - 1, z)), st = a.species(g.idx(x, y + 1, z));
        float4 sk = a.species(g.idx(x, y, z - 1)), sf = a.species(g.idx(x, y, z + 1));
        float4 avg = make_float4((sl.x + sr.x + sb.x + st.x + sk.x + sf.x) / 6.0f, (sl.y + sr.y + sb.y + st.y + sk.y + sf.y) / 6.0f,
                                 (sl.z + sr.z + sb.z + st.z + sk.z + sf.z) / 6.0f, (sl.w + sr.w + sb.w + st.w + sk.w + sf.w) / 6.0f);
        species = fx_mix4(species, avg, fx_clamp(dt * FC(0.12), 0.0f, FC(0.06)));
    }

    // Source injection (shaders.ts:189-201); the sphere list replaces the burner.
    float firePower = fx_clamp(u[U_FIRE_POWER], FC(0.1), 4.0f);
    float powerRoot = sqrtf(firePower);
    float thermalPower = fx_min(powerRoot, 1.0f + FC(0.22) * (powerRoot - 1.0f));
    float source;
    if (P.emitter_mode == FIREX_EMITTER_SPHERES) {
        source = 0.0f;
        const float j = P.jitter;
        for (int s = 0; s < P.num_spheres; ++s) {
            const firex_sphere& sp = P.spheres[s];
            if (!fx_sphere_inside(sp, x, y, z)) continue;
            source = 1.0f;
            species.x = fx_max(species.x, sp.fuel * j);
            flow.w = fx_max(flow.w, u[U_T_AMBIENT] + (sp.temperature - u[U_T_AMBIENT]) * j);
        }
    } else {
        source = fx_burner(u, nx, ny, nz);
        species.x = fx_max(species.x, source * u[U_FUEL_RATE] * firePower);
        flow.w = fx_max(flow.w, u[U_T_AMBIENT] + source * 1180.0f * thermalPower);
    }
    {
        float swx = sinf(u[U_TIME] * FC(2.3) + nz * 22.0f);
        float swy = 0.0f;
        float swz = cosf(u[U_TIME] * FC(1.9) + nx * 25.0f);
        float s = source * dt * FC(0.11) * u[U_VORTICITY] * powerRoot;
        flow.x = flow.x + swx * s;
        flow.y = flow.y + swy * s;
        flow.z = flow.z + swz * s;
        flow.y += source * dt * FC(0.52) * fx_clamp(u[U_LIFT], 0.0f, 4.0f) * powerRoot;
    }

    if (x == 0 || x == X - 1 || z == 0 || z == Z - 1 || y == Y - 1) {  // shaders.ts:203-208
        species.y = fx_max(species.y, u[U_OXYGEN]);
        flow.w = fx_mix(flow.w, u[U_T_AMBIENT], FC(0.035));
    }

    // Liquid cooling and vapor (shaders.ts:212-215)
    float water = fx_clamp((float)a.liquid(id) * (1.0f / 4096.0f) * FC(3.4), 0.0f, 5.0f);
    float evaporation = water * fx_smoothstep(335.0f, 1040.0f, flow.w) * dt * FC(13.5);
    flow.w = fx_max(u[U_T_AMBIENT], flow.w - evaporation * 2080.0f - water * dt * 260.0f);
    species.w = fx_clamp(species.w + evaporation * FC(2.15), 0.0f, 3.0f);

    // O2 entrainment (shaders.ts:220-232)
    float entrainment = fx_clamp(u[U_ENTRAIN], 0.0f, 3.0f);
    float ambientOxygen = fx_max(u[U_OXYGEN], FC(0.001));
    float oxygenDeficit = fx_clamp((ambientOxygen - species.y) / ambientOxygen, 0.0f, 1.0f);
    float fuelCore = fx_smoothstep(FC(0.30), FC(0.78), species.x);
    float interfaceWeight = oxygenDeficit * fx_mix(1.0f, FC(0.18), fuelCore);
    float entrainmentMix = fx_clamp(dt * entrainment *
                                        (FC(0.12) + FC(0.28) * fx_length3(flow.x, flow.y, flow.z) +
                                         FC(0.22) * fx_smoothstep(400.0f, 1500.0f, flow.w)) *
                                        interfaceWeight,
                                    0.0f, FC(0.08));
    species.y = fx_mix(species.y, ambientOxygen, entrainmentMix);

    // Arrhenius burn bounded by the 1:4 fuel:O2 ratio (shaders.ts:234-256)
    float fuelBefore = fx_max(species.x, 0.0f);
    float oxygenBefore = fx_max(species.y, 0.0f);
    float availableFuel = fx_min(fuelBefore, oxygenBefore * FC(0.25));
    float safeFuel = fx_max(fuelBefore, FC(0.00001));
    float safeOxygen = fx_max(oxygenBefore, FC(0.00001));
    float activation = expf(-15000.0f / fx_max(flow.w, u[U_T_AMBIENT]));
    float arrhenius = fx_clamp(FC(2.5e6) * activation * powf(safeFuel, FC(-0.30)) * powf(safeOxygen, FC(1.30)), 0.0f, 80.0f);
    float ignition = fx_smoothstep(690.0f, 930.0f, flow.w);
    float requestedBurn = availableFuel * (1.0f - expf(-arrhenius * ignition * dt)) * expf(-water * 18.0f);
    float burn = fx_clamp(requestedBurn, 0.0f, availableFuel);
    float richness = fx_clamp(1.0f - oxygenBefore / fx_max(fuelBefore * 4.0f, FC(0.00001)), 0.0f, 1.0f);
    species.x = fx_max(0.0f, fuelBefore - burn);
    species.y = fx_max(0.0f, oxygenBefore - burn * 4.0f);
    species.z = fx_clamp(species.z + burn * (1.0f + richness * FC(1.8)), 0.0f, 3.0f);
    species.w = fx_clamp(species.w + burn * FC(0.62), 0.0f, 3.0f);
    flow.w += burn * (2150.0f + 1450.0f * u[U_HEAT_EFF]);
    float reaction = fx_clamp(burn / fx_max(dt, FC(0.0001)) * FC(0.22), 0.0f, 4.0f);

    {  // vorticity confinement: curl x grad(T) (shaders.ts:258-272)
        float cx = 0.5f * ((top.z - bottom.z) * metric.y - (front.y - back.y) * metric.z);
        float cy = 0.5f * ((front.x - back.x) * metric.z - (right.z - left.z) * metric.x);
        float cz = 0.5f * ((right.y - left.y) * metric.x - (top.x - bottom.x) * metric.y);
        float gx = 0.5f * ((right.w - left.w) * metric.x) + FC(0.00001);
        float gy = 0.5f * ((top.w - bottom.w) * metric.y) + FC(0.00001);
        float gz = 0.5f * ((front.w - back.w) * metric.z) + FC(0.00001);
        float gl = fx_length3(gx, gy, gz);
        gx = gx / gl;
        gy = gy / gl;
        gz = gz / gl;
        float vs = FC(0.00135) * u[U_VORTICITY] * dt;
        flow.x = flow.x + (gy * cz - gz * cy) * vs;
        flow.y = flow.y + (gz * cx - gx * cz) * vs;
        flow.z = flow.z + (gx * cy - gy * cx) * vs;
    }
    {  // height-enveloped turbulence (shaders.ts:274-285)
        float time = u[U_TIME];
        float hotPlume = fx_smoothstep(520.0f, 1650.0f, flow.w);
        float heightEnvelope = fx_smoothstep(FC(0.045), FC(0.15), ny) * (1.0f - fx_smoothstep(FC(0.80), 1.0f, ny));
        float ltx = sinf(ny * 31.0f + nz * 19.0f + time * FC(3.1)) + FC(0.45) * sinf(ny * 67.0f - time * FC(5.3));
        float lty = FC(0.12) * sinf(nx * 29.0f + nz * 23.0f - time * FC(4.1));
        float ltz = cosf(ny * 27.0f - nx * 21.0f + time * FC(2.7)) + FC(0.45) * cosf(ny * 59.0f + time * FC(4.7));
        float ts = (FC(0.075) + FC(0.16) * u[U_VORTICITY]) * hotPlume * heightEnvelope * dt;
        flow.x = flow.x + ltx * ts;
        flow.y = flow.y + lty * ts;
        flow.z = flow.z + ltz * ts;
    }
    {  // buoyancy (shaders.ts:287-288)
        float buoyancy = fx_clamp((flow.w - u[U_T_AMBIENT]) / 1500.0f, FC(-0.1), FC(1.2));
        flow.y += buoyancy * dt * FC(0.72) * fx_clamp(u[U_BUOYANCY], 0.0f, 4.0f);
    }
    species.z *= expf(-water * dt * FC(4.8));
    {  // spray momentum (shaders.ts:293-297)
        float3 ext = fx_extent(u);
        float ox = FC(0.035) * ext.x, oy = FC(0.50) * ext.y, oz = FC(0.5) * ext.z;
        float tx = FC(0.52) * ext.x, ty = u[U_AIM_HEIGHT] * ext.y, tz = FC(0.5) * ext.z;
        float dx = tx - ox, dy = ty - oy, dz = tz - oz;
        float l = fx_length3(dx, dy, dz);
        dx = dx / l;
        dy = dy / l;
        dz = dz / l;
        flow.x = flow.x + dx * water * dt * FC(0.82);
        flow.y = flow.y + dy * water * dt * FC(0.82);
        flow.z = flow.z + dz * water * dt * FC(0.82);
    }
    // radiation and decay (shaders.ts:299-304)
    float persistence = fx_clamp(u[U_PERSISTENCE], FC(0.4), 3.0f);
    float radiation = FC(5.67e-8) * (powf(u[U_T_AMBIENT], 4.0f) - powf(fx_max(flow.w, 0.0f), 4.0f)) / (1005.0f * persistence);
    flow.w = fx_max(u[U_T_AMBIENT], flow.w + dt * radiation);
    species.z *= expf(-dt * FC(0.075) / persistence);
    species.w *= expf(-dt * FC(0.14) / persistence);

    // open-top outflow (shaders.ts:308-321)
    float outflow = fx_smoothstep(FC(0.84), FC(0.995), ny);
    species.x *= 1.0f - outflow;
    float outflowDecay = expf(-outflow * dt * 15.0f / persistence);
    species.z *= outflowDecay;
    species.w *= outflowDecay;
    flow.w = fx_mix(flow.w, u[U_T_AMBIENT], outflow * FC(0.16) / persistence);
    reaction *= 1.0f - outflow;
    if (y == Y - 1) {
        species.x = 0.0f;
        species.z = 0.0f;
        species.w = 0.0f;
        flow.w = u[U_T_AMBIENT];
        reaction = 0.0f;
    }
    // walls and clamps (shaders.ts:323-339)
    if (x == 0 || x == X - 1) flow.x = 0.0f;
    if (z == 0 || z == Z - 1) flow.z = 0.0f;
    if (y == 0) flow.y = 0.0f;
    if (y == Y - 1) flow.y = fx_max(0.0f, flow.y);
    flow.x = fx_clamp(flow.x, FC(-1.4), FC(1.4));
    flow.y = fx_clamp(flow.y, FC(-1.4), FC(1.4));
    flow.z = fx_clamp(flow.z, FC(-1.4), FC(1.4));
    flow.w = fx_clamp(flow.w, u[U_T_AMBIENT], 2900.0f);
    species = make_float4(fx_clamp(species.x, 0.0f, 3.0f), fx_clamp(species.y, 0.0f, 3.0f),
                          fx_clamp(species.z, 0.0f, 3.0f), fx_clamp(species.w, 0.0f, 3.0f));
    FxCellOut o;
    o.flow = flow;
    o.species = species;
    o.reaction = reaction;
    return o;
}

// Jacobi stencil constants (shaders.ts:386-389): w = metric^2, denominator 2(wx+wy+wz).
struct FxJacobiConst {
    float wx, wy, wz, denom;
};
FXD FxJacobiConst fx_jacobi_const(const float* u) {
    float3 m = fx_metric(u);
    FxJacobiConst c;
    c.wx = m.x * m.x;
    c.wy = m.y * m.y;
    c.wz = m.z * m.z;
    c.denom = 2.0f * (c.wx + c.wy + c.wz);
    return c;
}

// One Jacobi update from the six neighbours (shaders.ts:390-402), same order of
// operations as the reference: ((wx*(l+r) + wy*(b+t)) + wz*(k+f) - div) / denom.
FXD float fx_jacobi_numerator(const FxJacobiConst& c, float l, float r, float b, float t, float k, float f, float div) {
    return __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(c.wx, __fadd_rn(l, r)), __fmul_rn(c.wy, __fadd_rn(b, t))),
                               __fmul_rn(c.wz, __fadd_rn(k, f))),
                     div);
}
FXD float fx_jacobi_update(const FxJacobiConst& c, float l, float r, float b, float t, float k, float f, float div) {
    return __fdiv_rn(fx_jacobi_numerator(c, l, r, b, t, k, f, div), c.denom);
}

// Division by a constant d > 0 given rcp = RN(1/d): Markstein's correction step
// (P. Markstein, "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990): q = RN(x*rcp), e = x - q*d exactly by one
// fused multiply-add, result RN(q + e*rcp). The theorem assumes no underflow, so the
// step is used for 2^-96 <= |x| <= FLT_MAX (the quotient stays normal for any d below
// 2^30); zeros (whose sign must survive) and tiny x take the IEEE division, and
// x = +-inf or NaN, whose IEEE quotient by a finite d > 0 is x itself, is returned. The
// engine enables this path for a given d only after checking on the device that it
// equals IEEE x/d for every float x.
FXD float fx_div_by_const(float x, float d, float rcp) {
    const float ax = fabsf(x);
    if (ax >= 1.2621774483536189e-29f && ax <= 3.402823466e38f) {  // 2^-96 .. FLT_MAX
        const float q = __fmul_rn(x, rcp);
        const float e = __fmaf_rn(-q, d, x);
        return __fmaf_rn(e, rcp, q);
    }
    return ax <= 3.402823466e38f ? __fdiv_rn(x, d) : x;
}
