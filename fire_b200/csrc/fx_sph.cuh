// fx_sph.cuh — SPH droplets and liquid deposition (FIREX_PARTICLE_WGSL, shaders.ts:514-825).
//
// A droplet is two float4: (position in the unit domain, age) and (velocity, mass). The
// passes precede simulate: density (shaders.ts:602-638) and integration
// (shaders.ts:640-736) loop over every other droplet in index order, as the reference
// does, so each sum has the reference's order; deposition (shaders.ts:738-824) adds
// 16.12 fixed-point liquid mass with integer atomics, exact in any order. Every
// expression keeps the reference's operation order (compiled without contraction).
// sin, cos, tan and exp are evaluated in double and rounded to float, as the oracle does:
// the hash fract(sin(x) * 43758.5453) turns one ulp of sin into 1e-3, so both sides must
// agree on them to agree on the droplets.
#pragma once

#include "fx_device.cuh"


namespace fxsph {

FXD float sinF(float x) { return (float)sin((double)x); }
FXD float cosF(float x) { return (float)cos((double)x); }
FXD float tanF(float x) { return (float)tan((double)x); }
FXD float expF(float x) { return (float)exp((double)x); }
FXD float fract(float x) { return x - floorf(x); }
FXD float hash11(float v) { return fract(sinF(v * 12.9898f + 1.317f) * 43758.5453f); }
FXD float3 add(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
FXD float3 sub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
FXD float3 mul(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
FXD float3 muls(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
FXD float3 divv(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
FXD float3 divs(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
FXD float len(float3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
FXD float3 norm(float3 a) { return divs(a, len(a)); }
FXD float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
FXD float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }

struct Ctx {
    const float* u;
    int X, Y, Z;
    FXD float3 ext() const { return make_float3(fx_max(u[32], 0.001f), fx_max(u[33], 0.001f), fx_max(u[34], 0.001f)); }
    FXD bool spray() const { return u[26] >= 0.5f; }  // controls.z: nozzle type
};
FXD float3 nozzleOrigin() { return make_float3(0.035f, 0.50f, 0.5f); }
FXD float3 nozzleDirection(const Ctx& c) {
    const float3 target = make_float3(0.52f, fx_clamp(c.u[25], 0.08f, 0.82f), 0.5f);
    return norm(mul(sub(target, nozzleOrigin()), c.ext()));
}
// spawnParticle (shaders.ts:575-600)
FXD void spawn(const Ctx& c, unsigned id, float cycle, float4& pa, float4& vm) {
    const float seed = (float)id * 3.771f + cycle * 19.173f;
    const float radialRandom = sqrtf(hash11(seed + 0.17f));
    const float angularRandom = hash11(seed + 4.91f) * 6.2831853f;
    const float speedRandom = hash11(seed + 9.37f);
    const float3 direction = nozzleDirection(c);
    const float3 tangent = norm(cross(direction, make_float3(0.0f, 0.0f, 1.0f)));
    const float3 bitangent = norm(cross(direction, tangent));
    const float3 disk = add(muls(tangent, cosF(angularRandom)), muls(bitangent, sinF(angularRandom)));
    const float spread = c.spray() ? 0.72f : 0.10f;
    const float cone = tanF(fx_clamp(c.u[13], 0.005f, 0.78f)) * radialRandom * spread;
    const float3 launch = norm(add(direction, muls(disk, cone)));
    const float originRadius = c.spray() ? 0.006f : 0.0028f;
    const float3 origin = add(nozzleOrigin(), divv(muls(muls(disk, radialRandom), originRadius), c.ext()));
    const float sv = c.spray() ? 0.24f : 0.05f;
    const float speed = (0.82f + c.u[12] * 0.82f) * mixf(1.0f - sv * 0.5f, 1.0f + sv * 0.5f, speedRandom);
    const float3 v = muls(launch, speed);
    pa = make_float4(origin.x, origin.y, origin.z, 0.0f);
    vm = make_float4(v.x, v.y, v.z, 0.52f + c.u[12] * 0.88f);
}
FXD int cellIndex(const Ctx& c, int x, int y, int z) {
    x = min(max(x, 0), c.X - 1);
    y = min(max(y, 0), c.Y - 1);
    z = min(max(z, 0), c.Z - 1);
    return x + c.X * (y + c.Y * z);
}

// One warp per droplet. Lane l tests neighbour base + l of each run of 32; the warp then
// adds the terms of the neighbours in range in index order (ballot, then one shuffle per
// term), so every sum has the reference's order and rounding while the distance tests run
// 32 wide. Every lane ends with the same sums.
#define FX_FULL_MASK 0xffffffffu

// computeParticleDensity for droplet i (shaders.ts:602-638); p: 2 float4 per droplet
FXD float4 density_warp(const Ctx& c, int n, const float4* __restrict__ p, int i, int lane) {
    const float4 pa = __ldg(p + 2 * i), vm = __ldg(p + 2 * i + 1);
    if (vm.w <= 0.0001f) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float3 ext = c.ext();
    const float r = c.spray() ? 0.060f : 0.038f;
    float de = 0.0f, near = 0.0f;
    for (int base = 0; base < n; base += 32) {
        const int j = base + lane;
        float w = 0.0f;
        bool hit = false;
        if (j < n && j != i) {
            const float4 qa = __ldg(p + 2 * j), qm = __ldg(p + 2 * j + 1);
            if (!(qm.w <= 0.0001f)) {
                const float dist = len(mul(sub(make_float3(pa.x, pa.y, pa.z), make_float3(qa.x, qa.y, qa.z)), ext));
                if (dist > 0.00001f && dist < r) {
                    w = 1.0f - dist / r;
                    hit = true;
                }
            }
        }
        const float w2 = w * w, w3 = w * w * w;
        for (unsigned m = __ballot_sync(FX_FULL_MASK, hit); m; m &= m - 1) {
            const int src = __ffs(m) - 1;
            de += __shfl_sync(FX_FULL_MASK, w2, src);
            near += __shfl_sync(FX_FULL_MASK, w3, src);
        }
    }
    const float rest = 2.7f + c.u[12] * 0.9f;
    return make_float4(de, near, fx_max(de - rest, 0.0f) * 0.055f, near * 0.065f);
}

// integrateParticles for droplet i (shaders.ts:640-736); flow: the canonical flow field
FXD void integrate_warp(const Ctx& c, int n, const float4* __restrict__ p, const float4* __restrict__ dens,
                        const float4* __restrict__ flow, int i, int lane, float4& oa, float4& om) {
    const float4 pa = __ldg(p + 2 * i), vm = __ldg(p + 2 * i + 1);
    const float dt = c.u[4];
    if (dt <= 0.0f) {
        oa = pa;
        om = vm;
        return;
    }
    const bool waterOn = c.u[14] >= 0.5f && c.u[12] > 0.001f;
    if (vm.w <= 0.0001f) {
        const float wait = pa.w + dt;
        if (waterOn && wait >= 0.0f) {
            spawn(c, (unsigned)i, wait + c.u[6], oa, om);
        } else {
            const float3 no = nozzleOrigin();
            oa = make_float4(no.x, no.y, no.z, wait > 0.0f ? -0.72f : wait);
            om = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        return;
    }
    const float lifetime = 0.88f + hash11((float)i * 2.31f + 7.0f) * 0.52f;
    const float nextAge = pa.w + dt;
    const bool outside = pa.x < -0.03f || pa.y < -0.03f || pa.z < -0.03f || pa.x > 1.03f || pa.y > 1.03f || pa.z > 1.03f;
    if (nextAge >= lifetime || outside) {
        if (waterOn) {
            spawn(c, (unsigned)i, nextAge + c.u[6], oa, om);
        } else {
            const float3 no = nozzleOrigin();
            oa = make_float4(no.x, no.y, no.z, -hash11((float)i * 8.17f) * 0.72f);
            om = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        return;
    }
    const float3 ext = c.ext();
    const float r = c.spray() ? 0.060f : 0.038f;
    const float3 pos = make_float3(pa.x, pa.y, pa.z);
    float3 vel = make_float3(vm.x, vm.y, vm.z);
    const float4 pd = __ldg(dens + i);
    float3 pacc = make_float3(0.0f, 0.0f, 0.0f), vacc = pacc;
    for (int base = 0; base < n; base += 32) {
        const int j = base + lane;
        float3 tp = make_float3(0.0f, 0.0f, 0.0f), tv = tp;
        bool hit = false;
        if (j < n && j != i) {
            const float4 qa = __ldg(p + 2 * j), qm = __ldg(p + 2 * j + 1);
            if (!(qm.w <= 0.0001f)) {
                const float3 sep = mul(sub(pos, make_float3(qa.x, qa.y, qa.z)), ext);
                const float dist = len(sep);
                if (dist > 0.00001f && dist < r) {
                    const float w = 1.0f - dist / r;
                    const float3 dir = divs(sep, dist);
                    const float4 nd = __ldg(dens + j);
                    const float pr = (pd.z + nd.z) * w;
                    const float npr = (pd.w + nd.w) * w * w;
                    tp = muls(dir, pr + npr);
                    tv = muls(sub(make_float3(qm.x, qm.y, qm.z), vel), w * 0.018f);
                    hit = true;
                }
            }
        }
        for (unsigned m = __ballot_sync(FX_FULL_MASK, hit); m; m &= m - 1) {
            const int src = __ffs(m) - 1;
            pacc.x += __shfl_sync(FX_FULL_MASK, tp.x, src);
            pacc.y += __shfl_sync(FX_FULL_MASK, tp.y, src);
            pacc.z += __shfl_sync(FX_FULL_MASK, tp.z, src);
            vacc.x += __shfl_sync(FX_FULL_MASK, tv.x, src);
            vacc.y += __shfl_sync(FX_FULL_MASK, tv.y, src);
            vacc.z += __shfl_sync(FX_FULL_MASK, tv.z, src);
        }
    }
    // sampleFlow: nearest cell of the canonical flow
    const int cx = (int)(fx_clamp(pos.x, 0.0f, 0.99999f) * c.u[0]);
    const int cy = (int)(fx_clamp(pos.y, 0.0f, 0.99999f) * c.u[1]);
    const int cz = (int)(fx_clamp(pos.z, 0.0f, 0.99999f) * c.u[2]);
    const float4 g = __ldg(flow + cellIndex(c, cx, cy, cz));
    const float heat = fx_smoothstep(380.0f, 1500.0f, g.w);
    float3 acc = make_float3(0.0f, -0.58f, 0.0f);
    acc = add(acc, muls(sub(make_float3(g.x, g.y, g.z), vel), 0.30f + heat * 0.18f));
    const float disp = c.spray() ? 1.0f : 0.055f;
    const float coh = c.spray() ? 1.0f : 2.2f;
    acc = add(acc, add(muls(pacc, disp), muls(vacc, coh)));
    vel = add(vel, muls(acc, dt));
    float3 next = add(pos, divv(muls(vel, dt), ext));
    if (next.y < 0.012f) {
        next.y = 0.012f;
        vel.y = fabsf(vel.y) * 0.18f;
        vel = make_float3(vel.x * 0.72f, vel.y, vel.z * 0.72f);
    }
    if (next.x < 0.008f || next.x > 0.992f) {
        next.x = fx_clamp(next.x, 0.008f, 0.992f);
        vel.x *= -0.24f;
    }
    if (next.z < 0.008f || next.z > 0.992f) {
        next.z = fx_clamp(next.z, 0.008f, 0.992f);
        vel.z *= -0.24f;
    }
    const float mass = vm.w * expF(-heat * dt * 0.34f);
    oa = make_float4(next.x, next.y, next.z, nextAge);
    om = make_float4(fx_clamp(vel.x, -2.0f, 2.0f), fx_clamp(vel.y, -2.0f, 2.0f), fx_clamp(vel.z, -2.0f, 2.0f), mass);
}

// depositParticles (shaders.ts:738-824): integer sums, exact in any order, so the corners
// of a footprint go to separate lanes (8 trilinear corners for the jet, 27 cells for the
// spray, whose normalising total is added in the reference's z, y, x order by shuffles).
FXD void corner(const Ctx& c, uint32_t* liq, int x, int y, int z, float weight, float mass) {
    const uint32_t fixed = (uint32_t)fx_clamp(weight * mass * 4096.0f, 0.0f, 65535.0f);
    atomicAdd(liq + cellIndex(c, x, y, z), fixed);
}
FXD void depositAt_warp(const Ctx& c, uint32_t* liq, float3 position, float mass, int lane) {
    const float3 vp = sub(mul(position, make_float3(c.u[0], c.u[1], c.u[2])), make_float3(0.5f, 0.5f, 0.5f));
    if (!c.spray()) {
        if (lane >= 8) return;
        const int dx = lane & 1, dy = (lane >> 1) & 1, dz = lane >> 2;
        const float3 f = make_float3(fract(vp.x), fract(vp.y), fract(vp.z));
        const float3 iv = make_float3(1.0f - f.x, 1.0f - f.y, 1.0f - f.z);
        const float weight = (dx ? f.x : iv.x) * (dy ? f.y : iv.y) * (dz ? f.z : iv.z);
        corner(c, liq, (int)floorf(vp.x) + dx, (int)floorf(vp.y) + dy, (int)floorf(vp.z) + dz, weight, mass * 0.20f);
        return;
    }
    const int cx = (int)rintf(vp.x), cy = (int)rintf(vp.y), cz = (int)rintf(vp.z);
    const int ox = lane % 3 - 1, oy = (lane / 3) % 3 - 1, oz = lane / 9 - 1;  // lane = 9 (oz+1) + 3 (oy+1) + ox+1
    float kk = 0.0f;
    if (lane < 27) {
        const float d = len(sub(vp, make_float3((float)(cx + ox), (float)(cy + oy), (float)(cz + oz))));
        const float k = fx_max(0.0f, 1.0f - d * 0.52f);
        kk = k * k;
    }
    float total = 0.0f;
    for (int l = 0; l < 27; ++l) total += __shfl_sync(FX_FULL_MASK, kk, l);
    if (lane < 27) corner(c, liq, cx + ox, cy + oy, cz + oz, kk / fx_max(total, 0.0001f), mass);
}
// pa, pm: the droplet before the step; oa, om: after it
FXD void deposit_warp(const Ctx& c, float4 pa, float4 pm, float4 oa, float4 om, uint32_t* liq, int lane) {
    const float3 pos = make_float3(oa.x, oa.y, oa.z);
    const float mass = om.w;
    if (mass <= 0.0001f || pos.x < 0.0f || pos.y < 0.0f || pos.z < 0.0f || pos.x >= 1.0f || pos.y >= 1.0f || pos.z >= 1.0f)
        return;
    const float3 disp = sub(pos, make_float3(pa.x, pa.y, pa.z));
    const bool sweep = pm.w > 0.0001f && oa.w >= pa.w && len(mul(disp, c.ext())) < 0.20f;
    if (!sweep) {
        depositAt_warp(c, liq, pos, mass, lane);
        return;
    }
    for (unsigned k = 0; k < 3u; ++k) {
        const float fr = (float)k / 2.0f;
        depositAt_warp(c, liq, add(make_float3(pa.x, pa.y, pa.z), muls(disp, fr)), mass / 3.0f, lane);
    }
}

}  // namespace fxsph
