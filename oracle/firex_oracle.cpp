// firex_oracle.cpp — CPU restatement of the reference Fire-X simulation step.
//
// TEST INFRASTRUCTURE ONLY. This file is the correctness oracle for the CUDA library in
// fire_b200/ and the timed CPU baseline of bench.py. Nothing in the product links, loads
// or calls it; only tests/, __graft_entry__.smoke() and bench.py's CPU legs do.
//
// Parity status: the reference is WGSL run by WebGPU from TypeScript; neither a WebGPU
// implementation nor a JS runtime exists here, and the reference's own tests hold no
// numeric golden vectors for this path. The step is PINNED instead to the reference's own
// kernels executed on the CPU: tests/golden/wgsl_eval.py evaluates the WGSL text of
// shaders.ts:1-512 and pressureShaders.ts:1-161 in the dispatch order of
// FireXEngine.ts:2115-2276, and tests/test_reference_golden.py requires this restatement to
// reproduce those fixtures bit for bit (all three pressure branches, reset and developed
// states, dt = 0, 1/60, 1/30, a non-default parameter set, the SPH droplet passes of
// shaders.ts:514-825 with both nozzles and the spray switched off). The contracts the
// reference's tests assert are re-asserted by tests/test_oracle_contracts.py.
//
// Arithmetic conventions (shared with the CUDA kernels, which must match them):
//   * every WGSL expression is evaluated left to right in the precision T with no fused
//     multiply-add (compile with -ffp-contract=off);
//   * WGSL builtins follow the WGSL spec definitions: mix(a,b,t) = a*(1-t) + b*t,
//     smoothstep(e0,e1,x) = t*t*(3-2t) with t = clamp((x-e0)/(e1-e0),0,1),
//     fract(x) = x - floor(x), clamp(x,lo,hi) = min(max(x,lo),hi),
//     length(v) = sqrt(x*x + y*y + z*z), normalize(v) = v / length(v),
//     pow(x,y), sin, cos, exp from the C library in precision T;
//   * abstract-float literals are rounded from double to T (T(0.32));
//   * f32 -> f16 conversion rounds to nearest even (the f16 pressure branch).
//
// T = float restates the reference (f32 storage and math); T = double is the FP64
// accuracy oracle for the mixed-precision path.
#include "../include/firex.h"

// Oracle-only pressure branch for the precision study: branch A with the residual
// (correction) solve stored in FP16 as branch B stores it. The library does not offer it:
// measured against the FP64 step it misses the 1e-4 divergence bar by about 40x.
#define FXO_PRESSURE_WARM_F32_F16C 4
// Oracle-only pressure branch for the precision study: the primary (warm-started) solve
// stored in FP16 as branch B stores it, the divergence of the projected flow, the residual
// (correction) solve and the final projection in FP32 (iterative refinement of the FP16
// solve by the residual iterations).
#define FXO_PRESSURE_F16P_F32C 5

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace fxo {

template <typename T>
struct V3 {
    T x, y, z;
};
template <typename T>
struct V4 {
    T x, y, z, w;
};

// ---------------------------------------------------------------------------------------
// WGSL builtins (WGSL spec definitions; see header).
template <typename T>
static inline T clampT(T x, T lo, T hi) { return std::min(std::max(x, lo), hi); }
template <typename T>
static inline T mixT(T a, T b, T t) { return a * (T(1) - t) + b * t; }
template <typename T>
static inline T smoothstepT(T e0, T e1, T x) {
    T t = clampT((x - e0) / (e1 - e0), T(0), T(1));
    return t * t * (T(3) - T(2) * t);
}
template <typename T>
static inline T lengthT(V3<T> v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
template <typename T>
static inline V3<T> normalizeT(V3<T> v) {
    T l = lengthT(v);
    return {v.x / l, v.y / l, v.z / l};
}
template <typename T>
static inline V4<T> mix4(V4<T> a, V4<T> b, T t) {
    return {mixT(a.x, b.x, t), mixT(a.y, b.y, t), mixT(a.z, b.z, t), mixT(a.w, b.w, t)};
}
template <typename T>
static inline T sinT(T x) { return std::sin(x); }
template <typename T>
static inline T cosT(T x) { return std::cos(x); }
template <typename T>
static inline T expT(T x) { return std::exp(x); }
template <typename T>
static inline T powT(T x, T y) { return std::pow(x, y); }

// IEEE binary16 conversions written from the format definition (round to nearest even).
static inline uint16_t f32_to_f16(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t exp = (x >> 23) & 0xFFu;
    uint32_t man = x & 0x7FFFFFu;
    if (exp == 0xFFu) return (uint16_t)(sign | 0x7C00u | (man ? 0x200u : 0u));
    int e = (int)exp - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7C00u);  // overflow -> inf
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;  // underflows to signed zero
        man |= 0x800000u;
        int shift = 14 - e;  // 1 - e + 13
        uint32_t h = man >> shift;
        uint32_t rem = man & ((1u << shift) - 1u);
        uint32_t half = 1u << (shift - 1);
        if (rem > half || (rem == half && (h & 1u))) h += 1u;
        return (uint16_t)(sign | h);
    }
    uint32_t h = ((uint32_t)e << 10) | (man >> 13);
    uint32_t rem = man & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1u;  // may carry into exponent
    return (uint16_t)(sign | h);
}
static inline float f16_to_f32(uint16_t h) {
    uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1Fu;
    uint32_t man = h & 0x3FFu;
    uint32_t x;
    if (exp == 0) {
        if (man == 0) {
            x = sign;
        } else {
            int e = -1;
            do {
                e++;
                man <<= 1;
            } while ((man & 0x400u) == 0);
            man &= 0x3FFu;
            x = sign | ((uint32_t)(127 - 15 - e) << 23) | (man << 13);
        }
    } else if (exp == 31) {
        x = sign | 0x7F800000u | (man << 13);
    } else {
        x = sign | ((exp - 15 + 127) << 23) | (man << 13);
    }
    float f;
    std::memcpy(&f, &x, 4);
    return f;
}

// splitmix64 (Steele, Lea, Flood 2014): counter-based generator for the seeded extensions.
static inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
// Uniform float in [0, 1) with 24 random bits (exact in binary32).
static inline float unit24(uint64_t h) { return (float)(h >> 40) * (1.0f / 16777216.0f); }

// Initial velocity noise: component c of cell id, uniform in [-a, a].
static inline float velocity_noise(uint64_t seed, uint64_t cell, int comp, float a) {
    uint64_t h = splitmix64(splitmix64(seed ^ 0x6A09E667F3BCC909ull) + cell * 4u + (uint64_t)comp);
    float u = unit24(h);
    return a * (2.0f * u - 1.0f);
}
// Per-step emission jitter factor in [1-a, 1+a] for frame index f.
static inline float emission_jitter(uint64_t seed, int64_t frame, float a) {
    uint64_t h = splitmix64(splitmix64(seed ^ 0xBB67AE8584CAA73Bull) + (uint64_t)frame);
    float u = unit24(h);
    return 1.0f + a * (2.0f * u - 1.0f);
}

// ---------------------------------------------------------------------------------------
// Engine parameters: FireXEngine.parameters defaults (FireXEngine.ts:422-451) and the
// clamps of setParameter (FireXEngine.ts:937-1032). Values are JS numbers (f64) until
// writeUniforms stores them into a Float32Array.
struct Named {
    double burnerSize = 3.1, burnerDepth = 2.7, sourceThickness = 1.35, firePower = 2.5;
    double sourceLift = 1.6, buoyancyScale = 2.15, flamePersistence = 1.45, airEntrainment = 1.65;
    double fuelRate = 0.30, oxygenRate = 1, heatEfficiency = 0.86, vorticity = 3.6;
    double waterFlow = 0, sprayAngle = 10;
    bool waterEnabled = false;
    double cameraYaw = -0.34, cameraPitch = 0.03, cameraDistance = 4.9, viewMode = 0;
    double aimHeight = 0.42, nozzleType = 0, exposure = 1.25, frontDefinition = 1.65;
    double domainWidth = 1.15, domainHeight = 1.35, domainDepth = 1.15, viewZoom = 2.1;
    double opticalDetailTarget = 1024;
    bool displayImperial = false;
};

static inline double fin(double v, double fallback, int kind) {
    return (kind == FIREX_VALUE_NUMBER && std::isfinite(v)) ? v : fallback;
}
static inline double clampd(double v, double lo, double hi) { return std::max(lo, std::min(hi, v)); }

static void set_named(Named& p, const std::string& n, int kind, double v) {
    if (n == "burnerSize") p.burnerSize = clampd(fin(v, p.burnerSize, kind), 0.35, 3.2);
    else if (n == "burnerDepth") p.burnerDepth = clampd(fin(v, p.burnerDepth, kind), 0.35, 3.2);
    else if (n == "sourceThickness") p.sourceThickness = clampd(fin(v, p.sourceThickness, kind), 0.35, 2.5);
    else if (n == "firePower") p.firePower = clampd(fin(v, p.firePower, kind), 0.1, 4);
    else if (n == "sourceLift") p.sourceLift = clampd(fin(v, p.sourceLift, kind), 0, 4);
    else if (n == "buoyancyScale") p.buoyancyScale = clampd(fin(v, p.buoyancyScale, kind), 0, 4);
    else if (n == "flamePersistence") p.flamePersistence = clampd(fin(v, p.flamePersistence, kind), 0.4, 3);
    else if (n == "airEntrainment") p.airEntrainment = clampd(fin(v, p.airEntrainment, kind), 0, 3);
    else if (n == "fuelRate") p.fuelRate = fin(v, p.fuelRate, kind);
    else if (n == "oxygenRate") p.oxygenRate = fin(v, p.oxygenRate, kind);
    else if (n == "heatEfficiency") p.heatEfficiency = fin(v, p.heatEfficiency, kind);
    else if (n == "vorticity") p.vorticity = fin(v, p.vorticity, kind);
    else if (n == "waterFlow") p.waterFlow = fin(v, p.waterFlow, kind);
    else if (n == "sprayAngle") p.sprayAngle = fin(v, p.sprayAngle, kind);
    else if (n == "waterEnabled") { if (kind == FIREX_VALUE_BOOLEAN) p.waterEnabled = v != 0; }
    else if (n == "cameraYaw") p.cameraYaw = fin(v, p.cameraYaw, kind);
    else if (n == "cameraPitch") p.cameraPitch = fin(v, p.cameraPitch, kind);
    else if (n == "cameraDistance") p.cameraDistance = fin(v, p.cameraDistance, kind);
    else if (n == "viewMode") p.viewMode = clampd(std::round(fin(v, p.viewMode, kind)), 0, 7);
    else if (n == "aimHeight") p.aimHeight = clampd(fin(v, p.aimHeight, kind), 0.08, 0.82);
    else if (n == "nozzleType") p.nozzleType = fin(v, p.nozzleType, kind) >= 0.5 ? 1 : 0;
    else if (n == "exposure") p.exposure = clampd(fin(v, p.exposure, kind), 0.25, 3);
    else if (n == "frontDefinition") p.frontDefinition = clampd(fin(v, p.frontDefinition, kind), 0.5, 2.5);
    else if (n == "opticalDetailTarget") {
        double t = fin(v, p.opticalDetailTarget, kind);
        p.opticalDetailTarget = t >= 768 ? 1024 : t >= 384 ? 512 : t >= 192 ? 256 : 0;
    } else if (n == "domainWidth") p.domainWidth = clampd(fin(v, p.domainWidth, kind), 0.5, 4);
    else if (n == "domainHeight") p.domainHeight = clampd(fin(v, p.domainHeight, kind), 0.5, 6);
    else if (n == "domainDepth") p.domainDepth = clampd(fin(v, p.domainDepth, kind), 0.5, 4);
    else if (n == "displayImperial") p.displayImperial = (kind == FIREX_VALUE_BOOLEAN) ? v != 0 : fin(v, 0, kind) >= 0.5;
    else if (n == "viewZoom") p.viewZoom = clampd(fin(v, p.viewZoom, kind), 0.5, 5);
}

static bool get_named(const Named& p, const std::string& n, double* v) {
#define G(name) if (n == #name) { *v = (double)p.name; return true; }
    G(burnerSize) G(burnerDepth) G(sourceThickness) G(firePower) G(sourceLift) G(buoyancyScale)
    G(flamePersistence) G(airEntrainment) G(fuelRate) G(oxygenRate) G(heatEfficiency) G(vorticity)
    G(waterFlow) G(sprayAngle) G(waterEnabled) G(cameraYaw) G(cameraPitch) G(cameraDistance)
    G(viewMode) G(aimHeight) G(nozzleType) G(exposure) G(frontDefinition) G(domainWidth)
    G(domainHeight) G(domainDepth) G(viewZoom) G(opticalDetailTarget) G(displayImperial)
#undef G
    return false;
}

// writeUniforms (FireXEngine.ts:2043-2113): the 44-float block. Presentation-only entries
// (canvas aspect and size, ray steps) are written as 1, 1, 1, 0: the step does not read
// them; render.w is the particle count (:2069), which the particle passes read.
static void write_uniforms(float out[44], const Named& p, int X, int Y, int Z, double dt, double simTime,
                           int64_t frameIndex, int cinematic, int particles = 0) {
    double cells = (double)X * (double)Y * (double)Z;
    double v[44] = {(double)X, (double)Y, (double)Z, cells,
                    (double)dt, simTime, (double)frameIndex, (double)dt,
                    p.fuelRate, p.oxygenRate, p.heatEfficiency, p.vorticity,
                    p.waterFlow, (p.sprayAngle * M_PI) / 180, p.waterEnabled ? 1.0 : 0.0, 300,
                    p.cameraYaw, p.cameraPitch, p.cameraDistance, 1,
                    1, 1, 0, (double)particles,
                    p.viewMode, p.aimHeight, p.nozzleType, p.exposure,
                    p.burnerSize, p.burnerDepth, p.sourceThickness, p.firePower,
                    p.domainWidth, p.domainHeight, p.domainDepth, 0,
                    p.sourceLift, p.buoyancyScale, p.flamePersistence, p.viewZoom,
                    p.airEntrainment, p.frontDefinition, cinematic ? 1.0 : 0.0, p.opticalDetailTarget};
    for (int i = 0; i < 44; ++i) out[i] = (float)v[i];
}

// Extension block (no reference counterpart): emitter model and per-step jitter.
struct Ext {
    int emitterMode = FIREX_EMITTER_BURNER;
    float jitter = 1.0f;
    int numSpheres = 0;
    firex_sphere spheres[FIREX_MAX_SPHERES];
};

// ---------------------------------------------------------------------------------------
// The WGSL passes (shaders.ts:31-511, pressureShaders.ts:27-160), restated per cell.
template <typename T>
struct Grid {
    int X, Y, Z;
    size_t N;
    T u[44];  // uniform block converted to T
    Ext ext;
    // gridDimensions() -> vec3i(params.grid.xyz) (shaders.ts:31-33)
    // cellIndex with clamp (shaders.ts:43-51)
    inline size_t idx(int x, int y, int z) const {
        x = std::min(std::max(x, 0), X - 1);
        y = std::min(std::max(y, 0), Y - 1);
        z = std::min(std::max(z, 0), Z - 1);
        return (size_t)x + (size_t)X * ((size_t)y + (size_t)Y * (size_t)z);
    }
    // domainExtent() (shaders.ts:35-37)
    inline V3<T> extent() const {
        return {std::max(u[32], T(0.001)), std::max(u[33], T(0.001)), std::max(u[34], T(0.001))};
    }
    // cellMetric() = params.grid.xyz / domainExtent() (shaders.ts:39-41)
    inline V3<T> metric() const {
        V3<T> e = extent();
        return {u[0] / e.x, u[1] / e.y, u[2] / e.z};
    }
};

// trilinearFlow / trilinearSpecies (shaders.ts:61-95)
template <typename T>
static V4<T> trilinear(const Grid<T>& g, const V4<T>* f, V3<T> pos) {
    T dx = g.u[0], dy = g.u[1], dz = g.u[2];
    V3<T> sp = {clampT(pos.x - T(0.5), T(0), dx - T(1.001)), clampT(pos.y - T(0.5), T(0), dy - T(1.001)),
                clampT(pos.z - T(0.5), T(0), dz - T(1.001))};
    T flx = std::floor(sp.x), fly = std::floor(sp.y), flz = std::floor(sp.z);
    int bx = (int)flx, by = (int)fly, bz = (int)flz;
    T fx = sp.x - flx, fy = sp.y - fly, fz = sp.z - flz;
    V4<T> c000 = f[g.idx(bx, by, bz)], c100 = f[g.idx(bx + 1, by, bz)];
    V4<T> c010 = f[g.idx(bx, by + 1, bz)], c110 = f[g.idx(bx + 1, by + 1, bz)];
    V4<T> c001 = f[g.idx(bx, by, bz + 1)], c101 = f[g.idx(bx + 1, by, bz + 1)];
    V4<T> c011 = f[g.idx(bx, by + 1, bz + 1)], c111 = f[g.idx(bx + 1, by + 1, bz + 1)];
    V4<T> z0 = mix4(mix4(c000, c100, fx), mix4(c010, c110, fx), fy);
    V4<T> z1 = mix4(mix4(c001, c101, fx), mix4(c011, c111, fx), fy);
    return mix4(z0, z1, fz);
}

// emitter (shaders.ts:101-133)
template <typename T>
static T emitter(const Grid<T>& g, V3<T> np) {
    const T* u = g.u;
    T time = u[5];
    V3<T> ext = g.extent();
    V3<T> position = {np.x * ext.x, np.y * ext.y, np.z * ext.z};
    V3<T> center = {ext.x * T(0.5) + sinT(time * T(1.73)) * T(0.013), T(0.075),
                    ext.z * T(0.5) + cosT(time * T(1.37)) * T(0.011)};
    V3<T> off = {position.x - center.x, position.y - center.y, position.z - center.z};
    const T baseRadius = T(std::sqrt(0.02024));  // const-expression, evaluated in f64
    T radiusX = std::min(baseRadius * clampT(u[28], T(0.35), T(3.2)), ext.x * T(0.42));
    T radiusZ = std::min(baseRadius * clampT(u[29], T(0.35), T(3.2)), ext.z * T(0.42));
    T sourceThickness = clampT(u[30], T(0.35), T(2.5));
    T radial = off.x * off.x / (radiusX * radiusX) + off.z * off.z / (radiusZ * radiusZ);
    T vertical = off.y * off.y / (T(0.0022) * sourceThickness * sourceThickness);
    T cellular = T(0.76) + T(0.24) * sinT(position.x * T(49.0) + time * T(5.2)) *
                               sinT(position.z * T(43.0) - time * T(4.4));
    T lobeArg = sinT(off.x / std::max(radiusX, T(0.001)) * T(6.2) + time * T(1.7)) *
                sinT(off.z / std::max(radiusZ, T(0.001)) * T(5.4) - time * T(1.3));
    T cinematicLobes = mixT(T(0.48), T(1.18), smoothstepT(T(-0.42), T(0.48), lobeArg));
    T sourceTexture = mixT(cellular, cellular * cinematicLobes, clampT(u[42], T(0), T(1)));
    T pulse = T(0.84) + T(0.16) * sinT(time * T(3.7) + position.x * T(27.0) + position.z * T(21.0));
    return expT(-(radial + vertical)) * sourceTexture * pulse;
}

// Sphere emitter mask (extension): |c + 0.5 - center|^2 <= r^2 in float, fixed order.
static inline bool sphere_inside(const firex_sphere& s, int x, int y, int z) {
    float dx = ((float)x + 0.5f) - s.center[0];
    float dy = ((float)y + 0.5f) - s.center[1];
    float dz = ((float)z + 0.5f) - s.center[2];
    float d2 = (dx * dx + dy * dy) + dz * dz;
    return d2 <= s.radius * s.radius;
}

// simulate (shaders.ts:151-342). Writes flowOut, speciesOut and the reaction field.
template <typename T>
static void simulate_cell(const Grid<T>& g, int x, int y, int z, const V4<T>* flowIn, const V4<T>* speciesIn,
                          const uint32_t* liquid, V4<T>* flowOut, V4<T>* speciesOut, T* reactionOut) {
    const T* u = g.u;
    const int X = g.X, Y = g.Y, Z = g.Z;
    size_t id = g.idx(x, y, z);
    V3<T> dims = {u[0], u[1], u[2]};
    V3<T> pic = {T(x) + T(0.5), T(y) + T(0.5), T(z) + T(0.5)};
    V3<T> np = {pic.x / dims.x, pic.y / dims.y, pic.z / dims.z};
    T dt = u[4];

    V4<T> originalFlow = flowIn[id];
    V3<T> metric = g.metric();
    V3<T> backtrace = {pic.x - originalFlow.x * dt * metric.x, pic.y - originalFlow.y * dt * metric.y,
                       pic.z - originalFlow.z * dt * metric.z};
    V4<T> flow = trilinear(g, flowIn, backtrace);
    V4<T> species = trilinear(g, speciesIn, backtrace);
    species = {std::max(species.x, T(0)), std::max(species.y, T(0)), std::max(species.z, T(0)),
               std::max(species.w, T(0))};

    V4<T> left = flowIn[g.idx(x - 1, y, z)], right = flowIn[g.idx(x + 1, y, z)];
    V4<T> bottom = flowIn[g.idx(x, y - 1, z)], top = flowIn[g.idx(x, y + 1, z)];
    V4<T> back = flowIn[g.idx(x, y, z - 1)], front = flowIn[g.idx(x, y, z + 1)];

    V3<T> velAvg = {(left.x + right.x + bottom.x + top.x + back.x + front.x) / T(6.0),
                    (left.y + right.y + bottom.y + top.y + back.y + front.y) / T(6.0),
                    (left.z + right.z + bottom.z + top.z + back.z + front.z) / T(6.0)};
    T vmix = clampT(dt * T(0.32), T(0), T(0.12));
    flow.x = mixT(flow.x, velAvg.x, vmix);
    flow.y = mixT(flow.y, velAvg.y, vmix);
    flow.z = mixT(flow.z, velAvg.z, vmix);
    T tempAvg = (left.w + right.w + bottom.w + top.w + back.w + front.w) / T(6.0);
    flow.w = mixT(flow.w, tempAvg, clampT(dt * T(0.18), T(0), T(0.08)));

    V4<T> sl = speciesIn[g.idx(x - 1, y, z)], sr = speciesIn[g.idx(x + 1, y, z)];
    V4<T> sb = speciesIn[g.idx(x, y - 1, z)], st = speciesIn[g.idx(x, y + 1, z)];
    V4<T> sk = speciesIn[g.idx(x, y, z - 1)], sf = speciesIn[g.idx(x, y, z + 1)];
    V4<T> spAvg = {(sl.x + sr.x + sb.x + st.x + sk.x + sf.x) / T(6.0), (sl.y + sr.y + sb.y + st.y + sk.y + sf.y) / T(6.0),
                   (sl.z + sr.z + sb.z + st.z + sk.z + sf.z) / T(6.0), (sl.w + sr.w + sb.w + st.w + sk.w + sf.w) / T(6.0)};
    species = mix4(species, spAvg, clampT(dt * T(0.12), T(0), T(0.06)));

    // Source injection (shaders.ts:189-201); SPHERES replaces the burner (extension).
    T firePower = clampT(u[31], T(0.1), T(4.0));
    T powerRoot = std::sqrt(firePower);
    T thermalPower = std::min(powerRoot, T(1.0) + T(0.22) * (powerRoot - T(1.0)));
    T source;
    if (g.ext.emitterMode == FIREX_EMITTER_SPHERES) {
        source = T(0);
        T j = T(g.ext.jitter);
        for (int s = 0; s < g.ext.numSpheres; ++s) {
            const firex_sphere& sph = g.ext.spheres[s];
            if (!sphere_inside(sph, x, y, z)) continue;
            source = T(1);
            species.x = std::max(species.x, T(sph.fuel) * j);
            flow.w = std::max(flow.w, u[15] + (T(sph.temperature) - u[15]) * j);
        }
    } else {
        source = emitter(g, np);
        species.x = std::max(species.x, source * u[8] * firePower);
        flow.w = std::max(flow.w, u[15] + source * T(1180.0) * thermalPower);
    }
    V3<T> swirl = {sinT(u[5] * T(2.3) + np.z * T(22.0)), T(0.0), cosT(u[5] * T(1.9) + np.x * T(25.0))};
    T swirlScale = source * dt * T(0.11) * u[11] * powerRoot;
    flow.x = flow.x + swirl.x * swirlScale;
    flow.y = flow.y + swirl.y * swirlScale;
    flow.z = flow.z + swirl.z * swirlScale;
    flow.y += source * dt * T(0.52) * clampT(u[36], T(0.0), T(4.0)) * powerRoot;

    bool ambientBoundary = x == 0 || x == X - 1 || z == 0 || z == Z - 1 || y == Y - 1;
    if (ambientBoundary) {
        species.y = std::max(species.y, u[9]);
        flow.w = mixT(flow.w, u[15], T(0.035));
    }

    T water = clampT(T(liquid[id]) * (T(1.0) / T(4096.0)) * T(3.4), T(0.0), T(5.0));
    T evaporation = water * smoothstepT(T(335.0), T(1040.0), flow.w) * dt * T(13.5);
    flow.w = std::max(u[15], flow.w - evaporation * T(2080.0) - water * dt * T(260.0));
    species.w = clampT(species.w + evaporation * T(2.15), T(0.0), T(3.0));

    T entrainment = clampT(u[40], T(0.0), T(3.0));
    T ambientOxygen = std::max(u[9], T(0.001));
    T oxygenDeficit = clampT((ambientOxygen - species.y) / ambientOxygen, T(0.0), T(1.0));
    T fuelCore = smoothstepT(T(0.30), T(0.78), species.x);
    T interfaceWeight = oxygenDeficit * mixT(T(1.0), T(0.18), fuelCore);
    V3<T> fv = {flow.x, flow.y, flow.z};
    T entrainmentMix = clampT(dt * entrainment *
                                  (T(0.12) + T(0.28) * lengthT(fv) + T(0.22) * smoothstepT(T(400.0), T(1500.0), flow.w)) *
                                  interfaceWeight,
                              T(0.0), T(0.08));
    species.y = mixT(species.y, ambientOxygen, entrainmentMix);

    T fuelBefore = std::max(species.x, T(0.0));
    T oxygenBefore = std::max(species.y, T(0.0));
    T availableFuel = std::min(fuelBefore, oxygenBefore * T(0.25));
    T safeFuel = std::max(fuelBefore, T(0.00001));
    T safeOxygen = std::max(oxygenBefore, T(0.00001));
    T activation = expT(T(-15000.0) / std::max(flow.w, u[15]));
    T arrhenius = clampT(T(2.5e6) * activation * powT(safeFuel, T(-0.30)) * powT(safeOxygen, T(1.30)), T(0.0), T(80.0));
    T ignition = smoothstepT(T(690.0), T(930.0), flow.w);
    T requestedBurn = availableFuel * (T(1.0) - expT(-arrhenius * ignition * dt)) * expT(-water * T(18.0));
    T burn = clampT(requestedBurn, T(0.0), availableFuel);
    T richness = clampT(T(1.0) - oxygenBefore / std::max(fuelBefore * T(4.0), T(0.00001)), T(0.0), T(1.0));
    species.x = std::max(T(0.0), fuelBefore - burn);
    species.y = std::max(T(0.0), oxygenBefore - burn * T(4.0));
    species.z = clampT(species.z + burn * (T(1.0) + richness * T(1.8)), T(0.0), T(3.0));
    species.w = clampT(species.w + burn * T(0.62), T(0.0), T(3.0));
    flow.w += burn * (T(2150.0) + T(1450.0) * u[10]);
    T reaction = clampT(burn / std::max(dt, T(0.0001)) * T(0.22), T(0.0), T(4.0));

    V3<T> curl = {T(0.5) * ((top.z - bottom.z) * metric.y - (front.y - back.y) * metric.z),
                  T(0.5) * ((front.x - back.x) * metric.z - (right.z - left.z) * metric.x),
                  T(0.5) * ((right.y - left.y) * metric.x - (top.x - bottom.x) * metric.y)};
    V3<T> tg = {T(0.5) * ((right.w - left.w) * metric.x), T(0.5) * ((top.w - bottom.w) * metric.y),
                T(0.5) * ((front.w - back.w) * metric.z)};
    V3<T> gd = normalizeT(V3<T>{tg.x + T(0.00001), tg.y + T(0.00001), tg.z + T(0.00001)});
    T vscale = T(0.00135) * u[11] * dt;
    V3<T> cr = {gd.y * curl.z - gd.z * curl.y, gd.z * curl.x - gd.x * curl.z, gd.x * curl.y - gd.y * curl.x};
    flow.x = flow.x + cr.x * vscale;
    flow.y = flow.y + cr.y * vscale;
    flow.z = flow.z + cr.z * vscale;

    T time = u[5];
    T hotPlume = smoothstepT(T(520.0), T(1650.0), flow.w);
    T heightEnvelope = smoothstepT(T(0.045), T(0.15), np.y) * (T(1.0) - smoothstepT(T(0.80), T(1.0), np.y));
    V3<T> lt = {sinT(np.y * T(31.0) + np.z * T(19.0) + time * T(3.1)) + T(0.45) * sinT(np.y * T(67.0) - time * T(5.3)),
                T(0.12) * sinT(np.x * T(29.0) + np.z * T(23.0) - time * T(4.1)),
                cosT(np.y * T(27.0) - np.x * T(21.0) + time * T(2.7)) + T(0.45) * cosT(np.y * T(59.0) + time * T(4.7))};
    T turbulenceStrength = (T(0.075) + T(0.16) * u[11]) * hotPlume * heightEnvelope;
    T ts = turbulenceStrength * dt;
    flow.x = flow.x + lt.x * ts;
    flow.y = flow.y + lt.y * ts;
    flow.z = flow.z + lt.z * ts;

    T buoyancy = clampT((flow.w - u[15]) / T(1500.0), T(-0.1), T(1.2));
    flow.y += buoyancy * dt * T(0.72) * clampT(u[37], T(0.0), T(4.0));

    species.z *= expT(-water * dt * T(4.8));
    V3<T> ext = g.extent();
    V3<T> nozzleOrigin = {T(0.035) * ext.x, T(0.50) * ext.y, T(0.5) * ext.z};
    V3<T> sprayTarget = {T(0.52) * ext.x, u[25] * ext.y, T(0.5) * ext.z};
    V3<T> sprayMomentum = normalizeT(V3<T>{sprayTarget.x - nozzleOrigin.x, sprayTarget.y - nozzleOrigin.y,
                                           sprayTarget.z - nozzleOrigin.z});
    flow.x = flow.x + sprayMomentum.x * water * dt * T(0.82);
    flow.y = flow.y + sprayMomentum.y * water * dt * T(0.82);
    flow.z = flow.z + sprayMomentum.z * water * dt * T(0.82);

    T persistence = clampT(u[38], T(0.4), T(3.0));
    T radiation = T(5.67e-8) * (powT(u[15], T(4.0)) - powT(std::max(flow.w, T(0.0)), T(4.0))) / (T(1005.0) * persistence);
    flow.w = std::max(u[15], flow.w + dt * radiation);
    species.z *= expT(-dt * T(0.075) / persistence);
    species.w *= expT(-dt * T(0.14) / persistence);

    T outflow = smoothstepT(T(0.84), T(0.995), np.y);
    species.x *= T(1.0) - outflow;
    T outflowDecay = expT(-outflow * dt * T(15.0) / persistence);
    species.z *= outflowDecay;
    species.w *= outflowDecay;
    flow.w = mixT(flow.w, u[15], outflow * T(0.16) / persistence);
    reaction *= T(1.0) - outflow;
    if (y == Y - 1) {
        species.x = T(0.0);
        species.z = T(0.0);
        species.w = T(0.0);
        flow.w = u[15];
        reaction = T(0.0);
    }
    if (x == 0 || x == X - 1) flow.x = T(0.0);
    if (z == 0 || z == Z - 1) flow.z = T(0.0);
    if (y == 0) flow.y = T(0.0);
    if (y == Y - 1) flow.y = std::max(T(0.0), flow.y);
    flow.x = clampT(flow.x, T(-1.4), T(1.4));
    flow.y = clampT(flow.y, T(-1.4), T(1.4));
    flow.z = clampT(flow.z, T(-1.4), T(1.4));
    flow.w = clampT(flow.w, u[15], T(2900.0));
    species = {clampT(species.x, T(0.0), T(3.0)), clampT(species.y, T(0.0), T(3.0)), clampT(species.z, T(0.0), T(3.0)),
               clampT(species.w, T(0.0), T(3.0))};
    flowOut[id] = flow;
    speciesOut[id] = species;
    reactionOut[id] = reaction;
}

// computeDivergence (shaders.ts:344-364): backward differences.
template <typename T>
static inline T divergence_cell(const Grid<T>& g, const V4<T>* flow, int x, int y, int z) {
    V3<T> m = g.metric();
    V4<T> c = flow[g.idx(x, y, z)];
    T left = flow[g.idx(x - 1, y, z)].x;
    T bottom = flow[g.idx(x, y - 1, z)].y;
    T back = flow[g.idx(x, y, z - 1)].z;
    return (c.x - left) * m.x + (c.y - bottom) * m.y + (c.z - back) * m.z;
}

// loadPressure (shaders.ts:366-373): Dirichlet 0 above the open top, clamped elsewhere.
template <typename T, typename P>
static inline T load_p(const Grid<T>& g, const P* p, int x, int y, int z);
template <>
inline float load_p<float, float>(const Grid<float>& g, const float* p, int x, int y, int z) {
    return y >= g.Y ? 0.0f : p[g.idx(x, y, z)];
}
template <>
inline double load_p<double, double>(const Grid<double>& g, const double* p, int x, int y, int z) {
    return y >= g.Y ? 0.0 : p[g.idx(x, y, z)];
}
template <>
inline float load_p<float, uint16_t>(const Grid<float>& g, const uint16_t* p, int x, int y, int z) {
    return y >= g.Y ? 0.0f : f16_to_f32(p[g.idx(x, y, z)]);
}
template <>
inline double load_p<double, uint16_t>(const Grid<double>& g, const uint16_t* p, int x, int y, int z) {
    return y >= g.Y ? 0.0 : (double)f16_to_f32(p[g.idx(x, y, z)]);
}

template <typename T, typename P>
static inline P store_p(T v);
template <>
inline float store_p<float, float>(float v) { return v; }
template <>
inline double store_p<double, double>(double v) { return v; }
template <>
inline uint16_t store_p<float, uint16_t>(float v) { return f32_to_f16(v); }
template <>
inline uint16_t store_p<double, uint16_t>(double v) { return f32_to_f16((float)v); }

// One Jacobi sweep: solvePressureGlobal (shaders.ts:375-403); solvePressureTiled
// (:409-459) and solvePressureF16Tiled (pressureShaders.ts:62-117) evaluate the same
// expression in the same order from a shared-memory tile, so one restatement serves all
// three (P = uint16_t is the f16-storage variant).
template <typename T, typename P>
static void jacobi_sweep(const Grid<T>& g, const P* pin, const T* div, P* pout) {
    V3<T> m = g.metric();
    T wx = m.x * m.x, wy = m.y * m.y, wz = m.z * m.z;
    T denom = T(2.0) * (wx + wy + wz);
#pragma omp parallel for schedule(static)
    for (int z = 0; z < g.Z; ++z)
        for (int y = 0; y < g.Y; ++y)
            for (int x = 0; x < g.X; ++x) {
                size_t id = g.idx(x, y, z);
                if (y == g.Y - 1) {
                    pout[id] = store_p<T, P>(T(0.0));
                    continue;
                }
                T nb = wx * (load_p<T, P>(g, pin, x - 1, y, z) + load_p<T, P>(g, pin, x + 1, y, z)) +
                       wy * (load_p<T, P>(g, pin, x, y - 1, z) + load_p<T, P>(g, pin, x, y + 1, z)) +
                       wz * (load_p<T, P>(g, pin, x, y, z - 1) + load_p<T, P>(g, pin, x, y, z + 1));
                pout[id] = store_p<T, P>((nb - div[id]) / denom);
            }
}

// pressureGradient + projectVelocity (shaders.ts:461-501; F16 pressureShaders.ts:119-160).
template <typename T, typename P>
static inline V3<T> pressure_gradient(const Grid<T>& g, const P* p, int x, int y, int z, V3<T> m) {
    T c = load_p<T, P>(g, p, x, y, z);
    return {(load_p<T, P>(g, p, x + 1, y, z) - c) * m.x, (load_p<T, P>(g, p, x, y + 1, z) - c) * m.y,
            (load_p<T, P>(g, p, x, y, z + 1) - c) * m.z};
}

template <typename T, typename P>
static void project(const Grid<T>& g, const V4<T>* flowIn, const P* p, V4<T>* flowOut) {
    V3<T> m = g.metric();
#pragma omp parallel for schedule(static)
    for (int z = 0; z < g.Z; ++z)
        for (int y = 0; y < g.Y; ++y)
            for (int x = 0; x < g.X; ++x) {
                V3<T> gr = pressure_gradient(g, p, x, y, z, m);
                V4<T> f = flowIn[g.idx(x, y, z)];
                f = {f.x - gr.x, f.y - gr.y, f.z - gr.z, f.w};
                if (y == g.Y - 1) {
                    V4<T> b = flowIn[g.idx(x, y - 1, z)];
                    V3<T> gb = pressure_gradient(g, p, x, y - 1, z, m);
                    f = {b.x - gb.x, b.y - gb.y, b.z - gb.z, f.w};
                }
                if (x == 0 || x == g.X - 1) f.x = T(0.0);
                if (z == 0 || z == g.Z - 1) f.z = T(0.0);
                if (y == 0) f.y = T(0.0);
                if (y == g.Y - 1) f.y = std::max(T(0.0), f.y);
                flowOut[g.idx(x, y, z)] = f;
            }
}

template <typename T>
static void divergence_pass(const Grid<T>& g, const V4<T>* flow, T* div) {
#pragma omp parallel for schedule(static)
    for (int z = 0; z < g.Z; ++z)
        for (int y = 0; y < g.Y; ++y)
            for (int x = 0; x < g.X; ++x) div[g.idx(x, y, z)] = divergence_cell(g, flow, x, y, z);
}

template <typename T>
static void simulate_pass(const Grid<T>& g, const V4<T>* flowIn, const V4<T>* speciesIn, const uint32_t* liquid,
                          V4<T>* flowOut, V4<T>* speciesOut, T* reaction) {
#pragma omp parallel for schedule(static)
    for (int z = 0; z < g.Z; ++z)
        for (int y = 0; y < g.Y; ++y)
            for (int x = 0; x < g.X; ++x) simulate_cell(g, x, y, z, flowIn, speciesIn, liquid, flowOut, speciesOut, reaction);
}

// ---------------------------------------------------------------------------------------
// SPH droplets and liquid deposition (FIREX_PARTICLE_WGSL, shaders.ts:514-825), in f32 as
// the reference. A particle is 8 floats: position (domain-normalised), age, velocity, mass.
// sin, cos, tan and exp are evaluated in double and rounded to float (the CUDA path does
// the same): the hash fract(sin(x) * 43758.5453) amplifies one ulp of sin into 1e-3, so
// the two sides must agree on those to agree on the droplets.
namespace sph {
static inline float sinF(float x) { return (float)std::sin((double)x); }
static inline float cosF(float x) { return (float)std::cos((double)x); }
static inline float tanF(float x) { return (float)std::tan((double)x); }
static inline float expF(float x) { return (float)std::exp((double)x); }
static inline float fract(float x) { return x - std::floor(x); }
static inline float hash11(float v) { return fract(sinF(v * 12.9898f + 1.317f) * 43758.5453f); }
struct F3 {
    float x, y, z;
};
static inline F3 add(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline F3 mul(F3 a, F3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline F3 muls(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline F3 divv(F3 a, F3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
static inline F3 divs(F3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
static inline float len(F3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline F3 norm(F3 a) { return divs(a, len(a)); }
static inline F3 cross(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
static inline float maxf(float a, float b) { return a < b ? b : a; }
static inline float minf(float a, float b) { return b < a ? b : a; }
static inline float clampf(float x, float lo, float hi) { return minf(maxf(x, lo), hi); }
static inline float smoothstepf(float e0, float e1, float x) {
    float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
static inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }

struct Ctx {
    const float* u;  // uniform block
    int X, Y, Z;
    F3 ext() const { return {maxf(u[32], 0.001f), maxf(u[33], 0.001f), maxf(u[34], 0.001f)}; }
    bool spray() const { return u[26] >= 0.5f; }  // controls.z: nozzle type
};
static inline F3 nozzleOrigin() { return {0.035f, 0.50f, 0.5f}; }
static inline F3 nozzleDirection(const Ctx& c) {
    const F3 target = {0.52f, clampf(c.u[25], 0.08f, 0.82f), 0.5f};
    return norm(mul(sub(target, nozzleOrigin()), c.ext()));
}
// spawnParticle (shaders.ts:575-600)
static inline void spawn(const Ctx& c, unsigned id, float cycle, float* out) {
    const float seed = (float)id * 3.771f + cycle * 19.173f;
    const float radialRandom = std::sqrt(hash11(seed + 0.17f));
    const float angularRandom = hash11(seed + 4.91f) * 6.2831853f;
    const float speedRandom = hash11(seed + 9.37f);
    const F3 direction = nozzleDirection(c);
    const F3 tangent = norm(cross(direction, {0.0f, 0.0f, 1.0f}));
    const F3 bitangent = norm(cross(direction, tangent));
    const F3 disk = add(muls(tangent, cosF(angularRandom)), muls(bitangent, sinF(angularRandom)));
    const float spread = c.spray() ? 0.72f : 0.10f;
    const float cone = tanF(clampf(c.u[13], 0.005f, 0.78f)) * radialRandom * spread;
    const F3 launch = norm(add(direction, muls(disk, cone)));
    const float originRadius = c.spray() ? 0.006f : 0.0028f;
    const F3 origin = add(nozzleOrigin(), divv(muls(muls(disk, radialRandom), originRadius), c.ext()));
    const float sv = c.spray() ? 0.24f : 0.05f;
    const float speed = (0.82f + c.u[12] * 0.82f) * mixf(1.0f - sv * 0.5f, 1.0f + sv * 0.5f, speedRandom);
    out[0] = origin.x, out[1] = origin.y, out[2] = origin.z, out[3] = 0.0f;
    const F3 v = muls(launch, speed);
    out[4] = v.x, out[5] = v.y, out[6] = v.z, out[7] = 0.52f + c.u[12] * 0.88f;
}
static inline size_t cellIndex(const Ctx& c, int x, int y, int z) {
    x = std::min(std::max(x, 0), c.X - 1);
    y = std::min(std::max(y, 0), c.Y - 1);
    z = std::min(std::max(z, 0), c.Z - 1);
    return (size_t)x + (size_t)c.X * ((size_t)y + (size_t)c.Y * z);
}
// computeParticleDensity (shaders.ts:602-638)
static void density(const Ctx& c, int n, const float* pin, float* dens) {
    const F3 ext = c.ext();
    const float r = c.spray() ? 0.060f : 0.038f;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const float* p = pin + 8 * i;
        float* d = dens + 4 * i;
        if (p[7] <= 0.0001f) {
            d[0] = d[1] = d[2] = d[3] = 0.0f;
            continue;
        }
        float de = 0.0f, near = 0.0f;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            const float* q = pin + 8 * j;
            if (q[7] <= 0.0001f) continue;
            const float dist = len(mul(sub({p[0], p[1], p[2]}, {q[0], q[1], q[2]}), ext));
            if (dist > 0.00001f && dist < r) {
                const float w = 1.0f - dist / r;
                de += w * w;
                near += w * w * w;
            }
        }
        const float rest = 2.7f + c.u[12] * 0.9f;
        d[0] = de, d[1] = near, d[2] = maxf(de - rest, 0.0f) * 0.055f, d[3] = near * 0.065f;
    }
}
// integrateParticles (shaders.ts:640-736); flow: the canonical flow field, as float4
static void integrate(const Ctx& c, int n, const float* pin, const float* dens, const float* flow, float* pout) {
    const F3 ext = c.ext();
    const float dt = c.u[4];
    const bool waterOn = c.u[14] >= 0.5f && c.u[12] > 0.001f;
    const float r = c.spray() ? 0.060f : 0.038f;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const float* p = pin + 8 * i;
        float* o = pout + 8 * i;
        if (dt <= 0.0f) {
            std::memcpy(o, p, 32);
            continue;
        }
        if (p[7] <= 0.0001f) {
            const float wait = p[3] + dt;
            if (waterOn && wait >= 0.0f) {
                spawn(c, (unsigned)i, wait + c.u[6], o);
            } else {
                const F3 no = nozzleOrigin();
                o[0] = no.x, o[1] = no.y, o[2] = no.z, o[3] = wait > 0.0f ? -0.72f : wait;
                o[4] = o[5] = o[6] = o[7] = 0.0f;
            }
            continue;
        }
        const float lifetime = 0.88f + hash11((float)i * 2.31f + 7.0f) * 0.52f;
        const float nextAge = p[3] + dt;
        const bool outside = p[0] < -0.03f || p[1] < -0.03f || p[2] < -0.03f || p[0] > 1.03f || p[1] > 1.03f || p[2] > 1.03f;
        if (nextAge >= lifetime || outside) {
            if (waterOn) {
                spawn(c, (unsigned)i, nextAge + c.u[6], o);
            } else {
                const F3 no = nozzleOrigin();
                o[0] = no.x, o[1] = no.y, o[2] = no.z, o[3] = -hash11((float)i * 8.17f) * 0.72f;
                o[4] = o[5] = o[6] = o[7] = 0.0f;
            }
            continue;
        }
        const F3 pos = {p[0], p[1], p[2]};
        F3 vel = {p[4], p[5], p[6]};
        const float* pd = dens + 4 * i;
        F3 pa = {0, 0, 0}, va = {0, 0, 0};
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            const float* q = pin + 8 * j;
            if (q[7] <= 0.0001f) continue;
            const F3 sep = mul(sub(pos, {q[0], q[1], q[2]}), ext);
            const float dist = len(sep);
            if (dist > 0.00001f && dist < r) {
                const float w = 1.0f - dist / r;
                const F3 dir = divs(sep, dist);
                const float* nd = dens + 4 * j;
                const float pr = (pd[2] + nd[2]) * w;
                const float npr = (pd[3] + nd[3]) * w * w;
                pa = add(pa, muls(dir, pr + npr));
                va = add(va, muls(sub({q[4], q[5], q[6]}, vel), w * 0.018f));
            }
        }
        // sampleFlow: nearest cell of the canonical flow
        const int cx = (int)(clampf(pos.x, 0.0f, 0.99999f) * c.u[0]);
        const int cy = (int)(clampf(pos.y, 0.0f, 0.99999f) * c.u[1]);
        const int cz = (int)(clampf(pos.z, 0.0f, 0.99999f) * c.u[2]);
        const float* g = flow + 4 * cellIndex(c, cx, cy, cz);
        const float heat = smoothstepf(380.0f, 1500.0f, g[3]);
        F3 acc = {0.0f, -0.58f, 0.0f};
        acc = add(acc, muls(sub({g[0], g[1], g[2]}, vel), 0.30f + heat * 0.18f));
        const float disp = c.spray() ? 1.0f : 0.055f;
        const float coh = c.spray() ? 1.0f : 2.2f;
        acc = add(acc, add(muls(pa, disp), muls(va, coh)));
        vel = add(vel, muls(acc, dt));
        F3 next = add(pos, divv(muls(vel, dt), ext));
        if (next.y < 0.012f) {
            next.y = 0.012f;
            vel.y = std::fabs(vel.y) * 0.18f;
            vel = {vel.x * 0.72f, vel.y, vel.z * 0.72f};
        }
        if (next.x < 0.008f || next.x > 0.992f) {
            next.x = clampf(next.x, 0.008f, 0.992f);
            vel.x *= -0.24f;
        }
        if (next.z < 0.008f || next.z > 0.992f) {
            next.z = clampf(next.z, 0.008f, 0.992f);
            vel.z *= -0.24f;
        }
        const float mass = p[7] * expF(-heat * dt * 0.34f);
        o[0] = next.x, o[1] = next.y, o[2] = next.z, o[3] = nextAge;
        o[4] = clampf(vel.x, -2.0f, 2.0f), o[5] = clampf(vel.y, -2.0f, 2.0f), o[6] = clampf(vel.z, -2.0f, 2.0f);
        o[7] = mass;
    }
}
// depositParticles (shaders.ts:738-824): 16.12 fixed-point liquid mass, integer sums
static inline void corner(const Ctx& c, uint32_t* liq, int x, int y, int z, float weight, float mass) {
    const uint32_t fixed = (uint32_t)clampf(weight * mass * 4096.0f, 0.0f, 65535.0f);
    liq[cellIndex(c, x, y, z)] += fixed;
}
static void deposit_at(const Ctx& c, uint32_t* liq, F3 position, float mass) {
    const F3 vp = sub(mul(position, {c.u[0], c.u[1], c.u[2]}), {0.5f, 0.5f, 0.5f});
    if (!c.spray()) {
        const int bx = (int)std::floor(vp.x), by = (int)std::floor(vp.y), bz = (int)std::floor(vp.z);
        const F3 f = {fract(vp.x), fract(vp.y), fract(vp.z)};
        const F3 iv = {1.0f - f.x, 1.0f - f.y, 1.0f - f.z};
        const float m = mass * 0.20f;
        corner(c, liq, bx, by, bz, iv.x * iv.y * iv.z, m);
        corner(c, liq, bx + 1, by, bz, f.x * iv.y * iv.z, m);
        corner(c, liq, bx, by + 1, bz, iv.x * f.y * iv.z, m);
        corner(c, liq, bx + 1, by + 1, bz, f.x * f.y * iv.z, m);
        corner(c, liq, bx, by, bz + 1, iv.x * iv.y * f.z, m);
        corner(c, liq, bx + 1, by, bz + 1, f.x * iv.y * f.z, m);
        corner(c, liq, bx, by + 1, bz + 1, iv.x * f.y * f.z, m);
        corner(c, liq, bx + 1, by + 1, bz + 1, f.x * f.y * f.z, m);
        return;
    }
    const int cx = (int)std::nearbyint(vp.x), cy = (int)std::nearbyint(vp.y), cz = (int)std::nearbyint(vp.z);
    float total = 0.0f;
    for (int oz = -1; oz <= 1; ++oz)
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) {
                const float d = len(sub(vp, {(float)(cx + ox), (float)(cy + oy), (float)(cz + oz)}));
                const float k = maxf(0.0f, 1.0f - d * 0.52f);
                total += k * k;
            }
    for (int oz = -1; oz <= 1; ++oz)
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) {
                const float d = len(sub(vp, {(float)(cx + ox), (float)(cy + oy), (float)(cz + oz)}));
                const float k = maxf(0.0f, 1.0f - d * 0.52f);
                corner(c, liq, cx + ox, cy + oy, cz + oz, k * k / maxf(total, 0.0001f), mass);
            }
}
static void deposit(const Ctx& c, int n, const float* pin, const float* pout, uint32_t* liq) {
    const F3 ext = c.ext();
    for (int i = 0; i < n; ++i) {
        const float* o = pout + 8 * i;
        const F3 pos = {o[0], o[1], o[2]};
        const float mass = o[7];
        if (mass <= 0.0001f || pos.x < 0.0f || pos.y < 0.0f || pos.z < 0.0f || pos.x >= 1.0f || pos.y >= 1.0f ||
            pos.z >= 1.0f)
            continue;
        const float* p = pin + 8 * i;
        const F3 disp = sub(pos, {p[0], p[1], p[2]});
        const bool sweep = p[7] > 0.0001f && o[3] >= p[3] && len(mul(disp, ext)) < 0.20f;
        if (!sweep) {
            deposit_at(c, liq, pos, mass);
            continue;
        }
        for (unsigned k = 0; k < 3u; ++k) {
            const float fr = (float)k / 2.0f;
            deposit_at(c, liq, add({p[0], p[1], p[2]}, muls(disp, fr)), mass / 3.0f);
        }
    }
}
// writeParticleInitialState (FireXEngine.ts:1976-2034): host double arithmetic, stored f32
static void initial_state(const Named& nm, int n, bool active, float* out) {
    const double aimX = (0.52 - 0.035) * nm.domainWidth;
    const double aimY = (nm.aimHeight - 0.5) * nm.domainHeight;
    const double aimLength = std::hypot(aimX, aimY);
    const double base[3] = {aimX / aimLength, aimY / aimLength, 0.0};
    const double tangent[3] = {base[1], -base[0], 0.0};
    auto hash = [](double v) {
        const double h = std::sin(v * 12.9898 + 1.317) * 43758.5453;
        return h - std::floor(h);
    };
    for (int i = 0; i < n; ++i) {
        float* o = out + 8 * i;
        const double phase = (double)i / n;
        const double angle = hash(i * 3.771 + 4.91) * M_PI * 2;
        const double radial = std::sqrt(hash(i * 3.771 + 0.17));
        const double spreadScale = nm.nozzleType >= 0.5 ? 0.72 : 0.1;
        const double cone = std::tan((nm.sprayAngle * M_PI) / 180) * radial * spreadScale;
        const double diskX = tangent[0] * std::cos(angle), diskY = tangent[1] * std::cos(angle), diskZ = -std::sin(angle);
        double dx = base[0] + diskX * cone, dy = base[1] + diskY * cone, dz = diskZ * cone;
        const double dl = std::sqrt(dx * dx + dy * dy + dz * dz);
        dx /= dl;
        dy /= dl;
        dz /= dl;
        const double sv = nm.nozzleType >= 0.5 ? 0.24 : 0.05;
        const double speed = (0.82 + nm.waterFlow * 0.82) * (1 - sv * 0.5 + hash(i * 3.771 + 9.37) * sv);
        const double age = phase * 0.72;
        const double originRadius = nm.nozzleType >= 0.5 ? 0.006 : 0.0028;
        o[0] = (float)(0.035 + (diskX * radial * originRadius + dx * speed * age) / nm.domainWidth);
        o[1] = (float)std::max(0.012, 0.5 + (diskY * radial * originRadius + dy * speed * age - 0.29 * age * age) / nm.domainHeight);
        o[2] = (float)(0.5 + (diskZ * radial * originRadius + dz * speed * age) / nm.domainDepth);
        o[3] = (float)(active ? age : -phase * 0.72);
        o[4] = (float)(active ? dx * speed : 0.0);
        o[5] = (float)(active ? dy * speed - 0.58 * age : 0.0);
        o[6] = (float)(active ? dz * speed : 0.0);
        o[7] = (float)(active ? 0.52 + nm.waterFlow * 0.88 : 0.0);
    }
}
}  // namespace sph

// ---------------------------------------------------------------------------------------
// The engine: resources (FireXEngine.ts:1573-1603), initializeFields (:1933-1974),
// encodeSimulationStep (:2115-2276).
struct SimBase {
    virtual ~SimBase() {}
    int X, Y, Z;
    size_t N;
    firex_options opt;
    Named named;
    int mode;  // resolved pressure branch
    double simulationTime = 0;
    int64_t frameIndex = 0;
    int speciesIndex = 0, pressureIndex = 0;
    std::string err;
    virtual void reset() = 0;
    virtual void step(double dt) = 0;
    virtual int read_field(int field, void* out, size_t bytes) = 0;
    virtual int write_field(int field, const void* in, size_t bytes) = 0;
    virtual void divergence_norm(double out[3]) = 0;
    // Divergence of the predicted flow (before the first projection) of the last step over
    // interior cells: L2, max abs, cell count. The accuracy metric of mixed precision
    // normalises divergence differences by this L2 norm of the FP64 step.
    double preDiv[3] = {0, 0, 0};
    // particles (8 floats each, ping-pong) and their density (4 floats each)
    int np = 0;
    std::vector<float> particles[2], pdensity;
    int particleIndex = 0;
    bool particleFieldActive = false, liquidMayContainWater = false;
    bool water_active() const { return named.waterEnabled && named.waterFlow > 0.001; }
    void write_particle_initial_state(bool active) {
        particles[0].assign((size_t)np * 8, 0.0f);
        sph::initial_state(named, np, active, particles[0].data());
        particles[1] = particles[0];
        particleIndex = 0;
        particleFieldActive = active;
    }
};

template <typename T>
struct Sim : SimBase {
    std::vector<V4<T>> flow[2], species[2];
    std::vector<T> pressure[2], correction[2], divergence, reaction;
    std::vector<uint16_t> pressure16[2], correction16[2];
    std::vector<uint32_t> liquid;
    int lastCorrection = 0;  // which correction buffer holds the last residual result
    bool lastCorrectionShared = false;

    void alloc() {
        for (int i = 0; i < 2; ++i) {
            flow[i].assign(N, V4<T>{0, 0, 0, 0});
            species[i].assign(N, V4<T>{0, 0, 0, 0});
            if (mode == FXO_PRESSURE_WARM_F32_F16C) {
                pressure[i].assign(N, T(0));
                correction16[i].assign(N, 0);
            } else if (mode == FXO_PRESSURE_F16P_F32C) {
                pressure16[i].assign(N, 0);
                correction[i].assign(N, T(0));
            } else if (mode == FIREX_PRESSURE_F16) {
                pressure16[i].assign(N, 0);
                correction16[i].assign(N, 0);
            } else {
                pressure[i].assign(N, T(0));
                if (mode == FIREX_PRESSURE_WARM_F32) correction[i].assign(N, T(0));
            }
        }
        divergence.assign(N, T(0));
        reaction.assign(N, T(0));
        liquid.assign(N, 0u);
    }

    Grid<T> grid(double dt) const {
        Grid<T> g;
        g.X = X;
        g.Y = Y;
        g.Z = Z;
        g.N = N;
        float u[44];
        write_uniforms(u, named, X, Y, Z, dt, simulationTime, frameIndex, opt.cinematic, np);
        for (int i = 0; i < 44; ++i) g.u[i] = T(u[i]);
        g.ext.emitterMode = opt.emitter_mode;
        g.ext.numSpheres = opt.num_spheres;
        for (int s = 0; s < FIREX_MAX_SPHERES; ++s) g.ext.spheres[s] = opt.spheres[s];
        g.ext.jitter = emission_jitter(opt.seed, frameIndex, opt.emission_jitter);
        return g;
    }

    void reset() override {
        pdensity.assign((size_t)np * 4, 0.0f);
        write_particle_initial_state(water_active());  // initializeFields (FireXEngine.ts:1972-1973)
        liquidMayContainWater = false;
        simulationTime = 0;
        frameIndex = 0;
        speciesIndex = 0;
        pressureIndex = 0;
        lastCorrection = 0;
        lastCorrectionShared = false;
        alloc();  // clearBuffer on every field
        // initializeFields kernel (shaders.ts:135-149): uniform holds only grid, oxygenRate
        // ([9]) and ambient 300 K ([15]) (FireXEngine.ts:1937-1946).
        float oxy = (float)named.oxygenRate;
        T o2 = std::max(T(oxy), T(0.0));
        for (size_t id = 0; id < N; ++id) {
            V4<T> f = {T(0), T(0), T(0), T(300.0f)};
            if (opt.velocity_noise > 0) {  // seeded velocity noise (extension)
                f.x = T(velocity_noise(opt.seed, id, 0, opt.velocity_noise));
                f.y = T(velocity_noise(opt.seed, id, 1, opt.velocity_noise));
                f.z = T(velocity_noise(opt.seed, id, 2, opt.velocity_noise));
            }
            flow[0][id] = f;
            species[0][id] = V4<T>{T(0), o2, T(0), T(0)};
        }
    }

    // The particle passes that precede simulate (FireXEngine.ts:2158-2171): droplets move
    // and deposit into the liquid field while water runs; when it stops, the liquid field is
    // cleared and the droplets return to their inactive initial state.
    void particle_pass(const Grid<T>& g) {
        if (water_active()) {
            if (!particleFieldActive) write_particle_initial_state(true);
            std::fill(liquid.begin(), liquid.end(), 0u);
            float u[44];
            for (int i = 0; i < 44; ++i) u[i] = (float)g.u[i];
            const sph::Ctx c{u, X, Y, Z};
            std::vector<float> conv;
            const float* flowf;
            if (std::is_same<T, float>::value) {
                flowf = reinterpret_cast<const float*>(flow[0].data());
            } else {
                conv.resize(N * 4);
                for (size_t i = 0; i < N; ++i) {
                    conv[4 * i] = (float)flow[0][i].x, conv[4 * i + 1] = (float)flow[0][i].y;
                    conv[4 * i + 2] = (float)flow[0][i].z, conv[4 * i + 3] = (float)flow[0][i].w;
                }
                flowf = conv.data();
            }
            const int pi = particleIndex;
            sph::density(c, np, particles[pi].data(), pdensity.data());
            sph::integrate(c, np, particles[pi].data(), pdensity.data(), flowf, particles[1 - pi].data());
            sph::deposit(c, np, particles[pi].data(), particles[1 - pi].data(), liquid.data());
            particleIndex = 1 - pi;
            liquidMayContainWater = true;
        } else if (liquidMayContainWater || particleFieldActive) {
            std::fill(liquid.begin(), liquid.end(), 0u);
            write_particle_initial_state(false);
            liquidMayContainWater = false;
        }
    }

    void step(double dt) override {
        Grid<T> g = grid(dt);
        particle_pass(g);
        int s = speciesIndex;
        simulate_pass(g, flow[0].data(), species[s].data(), liquid.data(), flow[1].data(), species[1 - s].data(),
                      reaction.data());
        speciesIndex = 1 - s;
        divergence_pass(g, flow[1].data(), divergence.data());
        interior_norm(divergence.data(), preDiv);
        const int P = opt.pressure_iterations, R = opt.correction_iterations;
        if (mode == FXO_PRESSURE_WARM_F32_F16C) {  // branch A, the residual solve stored as in branch B
            for (int i = 0; i < P; ++i) {
                jacobi_sweep<T, T>(g, pressure[pressureIndex].data(), divergence.data(), pressure[1 - pressureIndex].data());
                pressureIndex = 1 - pressureIndex;
            }
            project<T, T>(g, flow[1].data(), pressure[pressureIndex].data(), flow[0].data());
            divergence_pass(g, flow[0].data(), divergence.data());
            std::fill(correction16[0].begin(), correction16[0].end(), 0);
            std::fill(correction16[1].begin(), correction16[1].end(), 0);
            int ci = 0;
            for (int i = 0; i < R; ++i) {
                jacobi_sweep<T, uint16_t>(g, correction16[ci].data(), divergence.data(), correction16[1 - ci].data());
                ci = 1 - ci;
            }
            project<T, uint16_t>(g, flow[0].data(), correction16[ci].data(), flow[1].data());
            lastCorrection = ci;
            lastCorrectionShared = false;
        } else if (mode == FXO_PRESSURE_F16P_F32C) {  // FP16 primary solve, FP32 residual solve
            for (int i = 0; i < P; ++i) {
                jacobi_sweep<T, uint16_t>(g, pressure16[pressureIndex].data(), divergence.data(),
                                          pressure16[1 - pressureIndex].data());
                pressureIndex = 1 - pressureIndex;
            }
            project<T, uint16_t>(g, flow[1].data(), pressure16[pressureIndex].data(), flow[0].data());
            divergence_pass(g, flow[0].data(), divergence.data());
            std::fill(correction[0].begin(), correction[0].end(), T(0));
            std::fill(correction[1].begin(), correction[1].end(), T(0));
            int ci = 0;
            for (int i = 0; i < R; ++i) {
                jacobi_sweep<T, T>(g, correction[ci].data(), divergence.data(), correction[1 - ci].data());
                ci = 1 - ci;
            }
            project<T, T>(g, flow[0].data(), correction[ci].data(), flow[1].data());
            lastCorrection = ci;
            lastCorrectionShared = false;
        } else if (mode == FIREX_PRESSURE_WARM_F32) {  // branch A (FireXEngine.ts:2248-2273)
            for (int i = 0; i < P; ++i) {
                jacobi_sweep<T, T>(g, pressure[pressureIndex].data(), divergence.data(), pressure[1 - pressureIndex].data());
                pressureIndex = 1 - pressureIndex;
            }
            project<T, T>(g, flow[1].data(), pressure[pressureIndex].data(), flow[0].data());
            divergence_pass(g, flow[0].data(), divergence.data());
            std::fill(correction[0].begin(), correction[0].end(), T(0));
            std::fill(correction[1].begin(), correction[1].end(), T(0));
            int ci = 0;
            for (int i = 0; i < R; ++i) {
                jacobi_sweep<T, T>(g, correction[ci].data(), divergence.data(), correction[1 - ci].data());
                ci = 1 - ci;
            }
            project<T, T>(g, flow[0].data(), correction[ci].data(), flow[1].data());
            lastCorrection = ci;
            lastCorrectionShared = false;
        } else if (mode == FIREX_PRESSURE_F16) {  // branch B (FireXEngine.ts:2177-2213)
            for (int i = 0; i < P; ++i) {
                jacobi_sweep<T, uint16_t>(g, pressure16[pressureIndex].data(), divergence.data(),
                                          pressure16[1 - pressureIndex].data());
                pressureIndex = 1 - pressureIndex;
            }
            project<T, uint16_t>(g, flow[1].data(), pressure16[pressureIndex].data(), flow[0].data());
            divergence_pass(g, flow[0].data(), divergence.data());
            std::fill(correction16[0].begin(), correction16[0].end(), 0);
            std::fill(correction16[1].begin(), correction16[1].end(), 0);
            int ci = 0;
            for (int i = 0; i < R; ++i) {
                jacobi_sweep<T, uint16_t>(g, correction16[ci].data(), divergence.data(), correction16[1 - ci].data());
                ci = 1 - ci;
            }
            project<T, uint16_t>(g, flow[0].data(), correction16[ci].data(), flow[1].data());
            lastCorrection = ci;
            lastCorrectionShared = false;
        } else {  // branch C (FireXEngine.ts:2214-2246)
            std::fill(pressure[0].begin(), pressure[0].end(), T(0));
            std::fill(pressure[1].begin(), pressure[1].end(), T(0));
            pressureIndex = 0;
            for (int i = 0; i < P; ++i) {
                jacobi_sweep<T, T>(g, pressure[pressureIndex].data(), divergence.data(), pressure[1 - pressureIndex].data());
                pressureIndex = 1 - pressureIndex;
            }
            project<T, T>(g, flow[1].data(), pressure[pressureIndex].data(), flow[0].data());
            divergence_pass(g, flow[0].data(), divergence.data());
            std::fill(pressure[0].begin(), pressure[0].end(), T(0));
            std::fill(pressure[1].begin(), pressure[1].end(), T(0));
            int ci = 0;
            for (int i = 0; i < R; ++i) {
                jacobi_sweep<T, T>(g, pressure[ci].data(), divergence.data(), pressure[1 - ci].data());
                ci = 1 - ci;
            }
            project<T, T>(g, flow[0].data(), pressure[ci].data(), flow[1].data());
            lastCorrection = ci;
            lastCorrectionShared = true;
        }
        flow[0] = flow[1];  // copyFlow (shaders.ts:503-511)
        simulationTime += dt;
        frameIndex += 1;
    }

    template <typename E>
    int copy_out_vec4(const std::vector<V4<T>>& v, void* out, size_t bytes) {
        if (bytes != N * 16) return FIREX_ERR_BAD_ARG;
        float* o = (float*)out;
        for (size_t i = 0; i < N; ++i) {
            o[4 * i + 0] = (float)v[i].x;
            o[4 * i + 1] = (float)v[i].y;
            o[4 * i + 2] = (float)v[i].z;
            o[4 * i + 3] = (float)v[i].w;
        }
        return FIREX_OK;
    }
    int copy_out_scalar(const std::vector<T>& v, void* out, size_t bytes) {
        if (bytes != N * 4) return FIREX_ERR_BAD_ARG;
        float* o = (float*)out;
        for (size_t i = 0; i < N; ++i) o[i] = (float)v[i];
        return FIREX_OK;
    }
    int copy_out_half(const std::vector<uint16_t>& v, void* out, size_t bytes) {
        if (bytes != N * 4) return FIREX_ERR_BAD_ARG;
        float* o = (float*)out;
        for (size_t i = 0; i < N; ++i) o[i] = f16_to_f32(v[i]);
        return FIREX_OK;
    }

    int read_field(int field, void* out, size_t bytes) override {
        switch (field) {
            case FIREX_FIELD_FLOW: return copy_out_vec4<float>(flow[0], out, bytes);
            case FIREX_FIELD_SPECIES: return copy_out_vec4<float>(species[speciesIndex], out, bytes);
            case FIREX_FIELD_PRESSURE:
                if (mode == FIREX_PRESSURE_F16 || mode == FXO_PRESSURE_F16P_F32C)
                    return copy_out_half(pressure16[pressureIndex], out, bytes);
                return copy_out_scalar(pressure[pressureIndex], out, bytes);
            case FIREX_FIELD_DIVERGENCE: return copy_out_scalar(divergence, out, bytes);
            case FIREX_FIELD_REACTION: return copy_out_scalar(reaction, out, bytes);
            case FIREX_FIELD_CORRECTION:
                if (mode == FIREX_PRESSURE_F16 || mode == FXO_PRESSURE_WARM_F32_F16C)
                    return copy_out_half(correction16[lastCorrection], out, bytes);
                if (lastCorrectionShared) return copy_out_scalar(pressure[lastCorrection], out, bytes);
                return copy_out_scalar(correction[lastCorrection], out, bytes);
            case FIREX_FIELD_LIQUID:
                if (bytes != N * 4) return FIREX_ERR_BAD_ARG;
                std::memcpy(out, liquid.data(), bytes);
                return FIREX_OK;
            case FIREX_FIELD_EMITTER_MASK: {
                if (bytes != N) return FIREX_ERR_BAD_ARG;
                uint8_t* o = (uint8_t*)out;
                for (int z = 0; z < Z; ++z)
                    for (int y = 0; y < Y; ++y)
                        for (int x = 0; x < X; ++x) {
                            uint8_t m = 0;
                            if (opt.emitter_mode == FIREX_EMITTER_SPHERES)
                                for (int s = 0; s < opt.num_spheres; ++s)
                                    if (sphere_inside(opt.spheres[s], x, y, z)) m = 1;
                            o[(size_t)x + (size_t)X * ((size_t)y + (size_t)Y * z)] = m;
                        }
                return FIREX_OK;
            }
            case FIREX_FIELD_FINAL_DIVERGENCE: {
                std::vector<T> d(N);
                Grid<T> g = grid(0.0);
                divergence_pass(g, flow[0].data(), d.data());
                return copy_out_scalar(d, out, bytes);
            }
            case FIREX_FIELD_RENDER_FLOW:
            case FIREX_FIELD_RENDER_CHEMISTRY:
            case FIREX_FIELD_RENDER_MEDIA:
                if (bytes != N * 8) return FIREX_ERR_BAD_ARG;
                render_pack(field - FIREX_FIELD_RENDER_FLOW, (uint16_t*)out);
                return FIREX_OK;
        }
        return FIREX_ERR_BAD_ARG;
    }

    // storePackedFields / packFields (qualityShaders.ts:37-75): the three rgba16float render
    // volumes of the canonical state, as FP16 bits (round to nearest even). which: 0 flow
    // (u, v, w, normalised T), 1 chemistry (species), 2 media (reaction, soot, liquid,
    // display value). In view 7 the display value is the post-projection divergence the
    // presentation computes from flow[0] (FireXEngine.ts:2588-2596), 0 on the outer shell.
    void render_pack(int which, uint16_t* out) {
        float u[44];
        write_uniforms(u, named, X, Y, Z, 0.0, simulationTime, frameIndex, opt.cinematic, np);
        const bool view7 = (unsigned)clampT(std::nearbyint(u[24]), 0.0f, 7.0f) == 7u;
        std::vector<T> d;
        if (view7) {
            d.resize(N);
            Grid<T> g = grid(0.0);
            divergence_pass(g, flow[0].data(), d.data());
        }
        const V4<T>* sp = species[speciesIndex].data();
        for (int z = 0; z < Z; ++z)
            for (int y = 0; y < Y; ++y)
                for (int x = 0; x < X; ++x) {
                    const size_t id = (size_t)x + (size_t)X * ((size_t)y + (size_t)Y * z);
                    const V4<T> f = flow[0][id];
                    const V4<T> sr = sp[id];
                    const V4<T> spc = {std::max(sr.x, T(0)), std::max(sr.y, T(0)), std::max(sr.z, T(0)), std::max(sr.w, T(0))};
                    const T reaction = clampT(this->reaction[id], T(0), T(4));
                    const T richness = clampT(spc.x / std::max(spc.x + spc.y * T(0.25), T(0.0001)), T(0), T(1));
                    const T soot = spc.z * smoothstepT(T(0.25), T(0.82), richness);
                    const T liq = T(float(liquid[id])) * T(3.4 / 4096.0);
                    const bool shell = x == 0 || y == 0 || z == 0 || x + 1 >= X || y + 1 >= Y || z + 1 >= Z;
                    T disp = std::max(std::max(reaction, soot),
                                      std::max(liq, std::max(spc.w, smoothstepT(T(420.0), T(700.0), f.w))));
                    if (view7) disp = shell ? T(0) : d[id];
                    T v[4];
                    if (which == 0) {
                        v[0] = f.x, v[1] = f.y, v[2] = f.z, v[3] = clampT((f.w - T(300.0)) / T(2600.0), T(0), T(1));
                    } else if (which == 1) {
                        v[0] = spc.x, v[1] = spc.y, v[2] = spc.z, v[3] = spc.w;
                    } else {
                        v[0] = reaction, v[1] = soot, v[2] = liq, v[3] = disp;
                    }
                    for (int k = 0; k < 4; ++k) out[4 * id + k] = f32_to_f16((float)v[k]);
                }
    }

    int write_vec4(std::vector<V4<T>>& v, const void* in, size_t bytes) {
        if (bytes != N * 16) return FIREX_ERR_BAD_ARG;
        const float* s = (const float*)in;
        for (size_t i = 0; i < N; ++i) v[i] = V4<T>{T(s[4 * i]), T(s[4 * i + 1]), T(s[4 * i + 2]), T(s[4 * i + 3])};
        return FIREX_OK;
    }
    int write_scalar(std::vector<T>& v, const void* in, size_t bytes) {
        if (bytes != N * 4) return FIREX_ERR_BAD_ARG;
        const float* s = (const float*)in;
        for (size_t i = 0; i < N; ++i) v[i] = T(s[i]);
        return FIREX_OK;
    }
    int write_half(std::vector<uint16_t>& v, const void* in, size_t bytes) {
        if (bytes != N * 4) return FIREX_ERR_BAD_ARG;
        const float* s = (const float*)in;
        for (size_t i = 0; i < N; ++i) v[i] = f32_to_f16(s[i]);
        return FIREX_OK;
    }

    int write_field(int field, const void* in, size_t bytes) override {
        switch (field) {
            case FIREX_FIELD_FLOW: return write_vec4(flow[0], in, bytes);
            case FIREX_FIELD_SPECIES: return write_vec4(species[speciesIndex], in, bytes);
            case FIREX_FIELD_PRESSURE:
                if (mode == FIREX_PRESSURE_F16 || mode == FXO_PRESSURE_F16P_F32C)
                    return write_half(pressure16[pressureIndex], in, bytes);
                return write_scalar(pressure[pressureIndex], in, bytes);
            case FIREX_FIELD_DIVERGENCE: return write_scalar(divergence, in, bytes);
            case FIREX_FIELD_REACTION: return write_scalar(reaction, in, bytes);
            case FIREX_FIELD_LIQUID:
                if (bytes != N * 4) return FIREX_ERR_BAD_ARG;
                std::memcpy(liquid.data(), in, bytes);
                return FIREX_OK;
        }
        return FIREX_ERR_BAD_ARG;
    }

    // L2 and max abs of a cell field over interior cells (the one-cell shell excluded).
    void interior_norm(const T* d, double out[3]) const {
        double ss = 0, mx = 0, n = 0;
        for (int z = 1; z < Z - 1; ++z)
            for (int y = 1; y < Y - 1; ++y)
                for (int x = 1; x < X - 1; ++x) {
                    const double v = (double)d[(size_t)x + (size_t)X * ((size_t)y + (size_t)Y * z)];
                    ss += v * v;
                    mx = std::max(mx, std::fabs(v));
                    n += 1;
                }
        out[0] = std::sqrt(ss);
        out[1] = mx;
        out[2] = n;
    }

    void divergence_norm(double out[3]) override {
        std::vector<T> d(N);
        Grid<T> g = grid(0.0);
        divergence_pass(g, flow[0].data(), d.data());
        double ss = 0, mx = 0, n = 0;
        for (int z = 1; z < Z - 1; ++z)
            for (int y = 1; y < Y - 1; ++y)
                for (int x = 1; x < X - 1; ++x) {
                    double v = (double)d[g.idx(x, y, z)];
                    ss += v * v;
                    mx = std::max(mx, std::fabs(v));
                    n += 1;
                }
        out[0] = std::sqrt(ss);
        out[1] = mx;
        out[2] = n;
    }
};

}  // namespace fxo

// ---------------------------------------------------------------------------------------
// C entry points (names mirror include/firex.h with the fxo_ prefix; precision selects
// the f32 restatement (32) or the FP64 accuracy oracle (64)).
using namespace fxo;

static std::string g_create_error;

extern "C" {

int fxo_create(int precision, const int32_t dims[3], const firex_options* opt, void** out) {
    *out = nullptr;
    if (!dims || !opt || dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0 || dims[0] % 4 || dims[1] % 4 || dims[2] % 4) {
        g_create_error = "grid axes must be positive multiples of 4";
        return FIREX_ERR_BAD_ARG;
    }
    if (opt->pressure_iterations < 0 || opt->correction_iterations < 0 || opt->num_spheres < 0 ||
        opt->num_spheres > FIREX_MAX_SPHERES) {
        g_create_error = "bad options";
        return FIREX_ERR_BAD_ARG;
    }
    SimBase* s;
    if (precision == 64) s = new Sim<double>();
    else s = new Sim<float>();
    s->X = dims[0];
    s->Y = dims[1];
    s->Z = dims[2];
    s->N = (size_t)dims[0] * dims[1] * dims[2];
    s->opt = *opt;
    s->np = std::max(0, opt->particle_count);
    int mode = opt->pressure_mode;
    if (mode == FIREX_PRESSURE_AUTO)
        mode = ((long long)s->N >= FIREX_HEAVY_GRID_CELL_THRESHOLD) ? FIREX_PRESSURE_F16 : FIREX_PRESSURE_WARM_F32;
    s->mode = mode;
    s->reset();
    *out = s;
    return FIREX_OK;
}

int fxo_destroy(void* h) {
    delete (SimBase*)h;
    return FIREX_OK;
}

int fxo_set_parameter(void* h, const char* name, int32_t kind, double value) {
    set_named(((SimBase*)h)->named, name, kind, value);
    return FIREX_OK;
}

int fxo_get_parameter(void* h, const char* name, double* value) {
    return get_named(((SimBase*)h)->named, name, value) ? FIREX_OK : FIREX_ERR_BAD_ARG;
}

int fxo_reset(void* h) {
    ((SimBase*)h)->reset();
    return FIREX_OK;
}

int fxo_step(void* h, int32_t n, double dt) {
    SimBase* s = (SimBase*)h;
    for (int i = 0; i < n; ++i) s->step(dt);
    return FIREX_OK;
}

int fxo_sync(void*) { return FIREX_OK; }  // the CPU oracle computes synchronously

int fxo_read_field(void* h, int32_t field, void* out, size_t bytes) {
    return ((SimBase*)h)->read_field(field, out, bytes);
}

int fxo_write_field(void* h, int32_t field, const void* in, size_t bytes) {
    return ((SimBase*)h)->write_field(field, in, bytes);
}

int fxo_get_state(void* h, firex_state* st) {
    SimBase* s = (SimBase*)h;
    st->simulation_time = s->simulationTime;
    st->frame_index = s->frameIndex;
    st->species_index = s->speciesIndex;
    st->pressure_index = s->pressureIndex;
    return FIREX_OK;
}

int fxo_set_state(void* h, const firex_state* st) {
    SimBase* s = (SimBase*)h;
    if ((st->species_index & ~1) || (st->pressure_index & ~1)) return FIREX_ERR_BAD_ARG;
    s->simulationTime = st->simulation_time;
    s->frameIndex = st->frame_index;
    s->speciesIndex = st->species_index;
    s->pressureIndex = st->pressure_index;
    return FIREX_OK;
}

int fxo_get_uniforms(void* h, double dt, float out[44]) {
    SimBase* s = (SimBase*)h;
    write_uniforms(out, s->named, s->X, s->Y, s->Z, dt, s->simulationTime, s->frameIndex, s->opt.cinematic, s->np);
    return FIREX_OK;
}

int fxo_divergence_norm(void* h, double out[3]) {
    ((SimBase*)h)->divergence_norm(out);
    return FIREX_OK;
}

int fxo_pressure_mode(void* h) { return ((SimBase*)h)->mode; }

// The current droplets (8 floats each: position, age, velocity, mass).
int fxo_read_particles(void* h, void* out, size_t bytes) {
    SimBase* s = (SimBase*)h;
    if (bytes != (size_t)s->np * 32) return FIREX_ERR_BAD_ARG;
    if (bytes) std::memcpy(out, s->particles[s->particleIndex].data(), bytes);
    return FIREX_OK;
}
int fxo_write_particles(void* h, const void* in, size_t bytes) {
    SimBase* s = (SimBase*)h;
    if (bytes != (size_t)s->np * 32) return FIREX_ERR_BAD_ARG;
    if (bytes) std::memcpy(s->particles[s->particleIndex].data(), in, bytes);
    return FIREX_OK;
}

int fxo_pre_projection_norm(void* h, double out[3]) {
    for (int i = 0; i < 3; ++i) out[i] = ((SimBase*)h)->preDiv[i];
    return FIREX_OK;
}

float fxo_emission_jitter(uint64_t seed, int64_t frame, float a) { return emission_jitter(seed, frame, a); }
float fxo_velocity_noise(uint64_t seed, uint64_t cell, int comp, float a) { return velocity_noise(seed, cell, comp, a); }
uint16_t fxo_f32_to_f16(float f) { return f32_to_f16(f); }
float fxo_f16_to_f32(uint16_t h) { return f16_to_f32(h); }

int fxo_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

const char* fxo_last_error(void* h) { return h ? ((SimBase*)h)->err.c_str() : g_create_error.c_str(); }

// Reference memory model (gridConfiguration.ts:98-112, 272-291).
uint64_t fxo_reference_memory_estimate(const int32_t dims[3], int64_t particles) {
    uint64_t cells = (uint64_t)dims[0] * dims[1] * dims[2];
    uint64_t per = cells >= (uint64_t)FIREX_HEAVY_GRID_CELL_THRESHOLD ? 108 : 116;
    return cells * per + (uint64_t)std::max<int64_t>(particles, 0) * 80 + 64ull * 64 * 64 * 4;
}

}  // extern "C"
