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

// ---- packed FP32 pairs (add/sub/mul/fma .rn.f32x2, Blackwell): each lane is rounded
// exactly as the scalar IEEE operation, so pairing changes no result bit.
typedef unsigned long long fx_f2;
FXD fx_f2 fx_pack2(float a, float b) {
    fx_f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
FXD float2 fx_unpack2(fx_f2 v) {
    float a, b;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
    return make_float2(a, b);
}
FXD fx_f2 fx_add2(fx_f2 a, fx_f2 b) {
    fx_f2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
FXD fx_f2 fx_sub2(fx_f2 a, fx_f2 b) {
    fx_f2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
FXD fx_f2 fx_mul2(fx_f2 a, fx_f2 b) {
    fx_f2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
FXD fx_f2 fx_fma2(fx_f2 a, fx_f2 b, fx_f2 c) {
    fx_f2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// Division by a constant d > 0 given rcp = RN(1/d): Markstein's correction step
// (P. Markstein, "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990): q = RN(x*rcp), e = x - q*d exactly by one
// fused multiply-add, result RN(q + e*rcp). The theorem assumes no underflow, so the
// step is used for 2^-96 <= |x| <= FLT_MAX (the quotient stays normal for any d below
// 2^30); zeros (whose sign must survive) are returned as they are, tiny x take the IEEE
// division, and x = +-inf or NaN, whose IEEE quotient by a finite d > 0 is x itself, is
// returned. fx_div_range takes an explicit range [lo, hi] of |x| (divisors below 1 need
// hi < FLT_MAX so that x * rcp cannot overflow). The engine enables this path for a
// given (d, lo, hi) only after checking on the device that it equals IEEE x/d for every
// float x.
//
// Out-of-range operands (tiny nonzero, |x| above the range, inf, NaN): kept out of line
// so that the common path is three instructions and a compare, not a predicated IEEE
// division.
static __device__ __noinline__ float fx_div_rare(float x, float d) { return fabsf(x) <= 3.402823466e38f ? __fdiv_rn(x, d) : x; }

FXD float fx_div_range(float x, float d, float rcp, float lo, float hi) {
    const float q = __fmul_rn(x, rcp);
    const float e = __fmaf_rn(-q, d, x);
    float r = __fmaf_rn(e, rcp, q);
    const float ax = fabsf(x);
    if (!(ax >= lo && ax <= hi)) r = (x == 0.0f) ? x : fx_div_rare(x, d);  // a zero keeps its sign
    return r;
}

FXD float fx_div_by_const(float x, float d, float rcp) { return fx_div_range(x, d, rcp, 1.2621774483536189e-29f, 3.402823466e38f); }

// x / c.d, by the checked constant-divisor path when the engine enabled it. A divisor the
// engine did not enable carries lo = +inf, so every x takes the IEEE division of
// fx_div_range's rare path (zeros keep their sign): one 16-byte load, no flag.
FXD float fx_divc(float x, const FxDivc& c) {
    const float4 v = *reinterpret_cast<const float4*>(&c);  // d, rcp, lo, hi
    return fx_div_range(x, v.x, v.y, v.z, v.w);
}

// smoothstep with its constant denominator e1 - e0 held in c.
FXD float fx_smoothstep_c(float e0, float x, const FxDivc& c) {
    float t = fx_clamp(fx_divc(x - e0, c), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

// trilinearFlow / trilinearSpecies (shaders.ts:61-95): 8-tap trilinear sample at
// position - 0.5, clamped to [0, dims - 1.001]. The clamp bounds floor() to
// [0, dims - 2], so base + 1 is always inside the grid and the reference's clamped tap
// addressing reduces to fixed offsets (the integer clamp below only guards addresses).
struct FxTri {
    int base;
    float fx, fy, fz;
};
FXD FxTri fx_tri_setup(const FxGrid& g, const float* u, float px, float py, float pz) {
    float sx = fx_clamp(px - 0.5f, 0.0f, u[U_GRID_X] - FC(1.001));
    float sy = fx_clamp(py - 0.5f, 0.0f, u[U_GRID_Y] - FC(1.001));
    float sz = fx_clamp(pz - 0.5f, 0.0f, u[U_GRID_Z] - FC(1.001));
    float flx = floorf(sx), fly = floorf(sy), flz = floorf(sz);
    const int bx = min(max((int)flx, 0), g.X - 2), by = min(max((int)fly, 0), g.Y - 2), bz = min(max((int)flz, 0), g.Z - 2);
    FxTri t;
    t.base = bx + g.X * (by + g.Y * bz);
    t.fx = sx - flx;
    t.fy = sy - fly;
    t.fz = sz - flz;
    return t;
}
template <class Load>
FXD float4 fx_trilinear(const FxGrid& g, const FxTri& t, Load load) {
    const int X = g.X, XY = g.X * g.Y, b = t.base;
    float4 c000 = load(b), c100 = load(b + 1), c010 = load(b + X), c110 = load(b + X + 1);
    float4 c001 = load(b + XY), c101 = load(b + XY + 1), c011 = load(b + XY + X), c111 = load(b + XY + X + 1);
    float4 z0 = fx_mix4(fx_mix4(c000, c100, t.fx), fx_mix4(c010, c110, t.fx), t.fy);
    float4 z1 = fx_mix4(fx_mix4(c001, c101, t.fx), fx_mix4(c011, c111, t.fx), t.fy);
    return fx_mix4(z0, z1, t.fz);
}

// ---- per-step tables ------------------------------------------------------------------------
// Terms of simulate that depend only on time and on one or two coordinates are computed
// once per step into a per-simulation table by fxk_step_tables, with the same device
// expressions the per-cell code would evaluate (so results are bit-identical):
//   uniform : exp(-dt*0.075/persistence), exp(-dt*0.14/persistence), pow(T_amb, 4), and
//             every other per-step constant of the cell update (metric, mixing weights,
//             fire power and its root, clamped controls, the spray direction)
//   x       : swirl z term, burner cellular/lobe/radial x terms
//   y       : height envelope, outflow, outflow decay, outflow mix, burner vertical term
//   z       : swirl x term, burner cellular/lobe/radial z terms
//   (y, z)  : turbulence x term     (x, z): turbulence y term, burner pulse
//   (x, y)  : turbulence z term
struct FxTabLayout {
    int x, y, z, ltx, lty, ltz, pulse, total;
};
enum {
    TU_DECAY_Z = 0, TU_DECAY_W, TU_TAMB4,
    TU_MX, TU_MY, TU_MZ,                           // metric (shaders.ts:39-41)
    TU_VMIX, TU_TMIX, TU_SMIX,                     // diffusion weights of velocity, T, species
    TU_POWER, TU_POWER_ROOT, TU_THERMAL,           // firePower, sqrt, thermal power
    TU_LIFT, TU_ENTRAIN, TU_AMB_O2, TU_HEAT,       // clamped lift, entrainment, ambient O2, heat release
    TU_VORT_S, TU_TURB, TU_BUOY, TU_CINE,          // vorticity step, turbulence gain, clamped buoyancy, cinematic
    TU_SPRAY_X, TU_SPRAY_Y, TU_SPRAY_Z,            // unit spray direction
    TU_COUNT = 24
};
enum { TX_SWZ = 0, TX_CELL = 1, TX_LOBE = 2, TX_RAD = 3, TX_COUNT = 4 };
enum { TY_HE = 0, TY_OUT = 1, TY_DECAY = 2, TY_MIX = 3, TY_VERT = 4, TY_COUNT = 5 };
enum { TZ_SWX = 0, TZ_CELL = 1, TZ_LOBE = 2, TZ_RAD = 3, TZ_COUNT = 4 };
__host__ __device__ inline FxTabLayout fx_tab_layout(int X, int Y, int Z) {
    FxTabLayout L;
    L.x = TU_COUNT;
    L.y = L.x + TX_COUNT * X;
    L.z = L.y + TY_COUNT * Y;
    L.ltx = L.z + TZ_COUNT * Z;
    L.lty = L.ltx + Y * Z;
    L.ltz = L.lty + X * Z;
    L.pulse = L.ltz + X * Y;
    L.total = L.pulse + X * Z;
    return L;
}

// Burner geometry shared by the table entries (emitter, shaders.ts:101-133).
struct FxBurnerGeom {
    float time, cx, cz, radiusX, radiusZ, thickness;
    float3 ext;
};
FXD FxBurnerGeom fx_burner_geom(const float* u) {
    FxBurnerGeom G;
    G.time = u[U_TIME];
    G.ext = fx_extent(u);
    G.cx = G.ext.x * 0.5f + sinf(G.time * FC(1.73)) * FC(0.013);
    G.cz = G.ext.z * 0.5f + cosf(G.time * FC(1.37)) * FC(0.011);
    const float baseRadius = FC(0.1422673539502299);  // sqrt(0.02024), a WGSL const-expression
    G.radiusX = fx_min(baseRadius * fx_clamp(u[U_BURNER_X], FC(0.35), FC(3.2)), G.ext.x * FC(0.42));
    G.radiusZ = fx_min(baseRadius * fx_clamp(u[U_BURNER_Z], FC(0.35), FC(3.2)), G.ext.z * FC(0.42));
    G.thickness = fx_clamp(u[U_THICKNESS], FC(0.35), FC(2.5));
    return G;
}

// Table entry i of a simulation whose uniform block is u.
FXD float fx_table_entry(const float* u, int X, int Y, int Z, int i) {
    const FxTabLayout L = fx_tab_layout(X, Y, Z);
    const float time = u[U_TIME], dt = u[U_DT];
    const float persistence = fx_clamp(u[U_PERSISTENCE], FC(0.4), 3.0f);
    auto nrm = [](int c, float dim) { return ((float)c + 0.5f) / dim; };
    if (i < L.x) {
        const float3 m = fx_metric(u);
        const float firePower = fx_clamp(u[U_FIRE_POWER], FC(0.1), 4.0f);
        const float powerRoot = sqrtf(firePower);
        switch (i) {
            case TU_DECAY_Z: return expf(-dt * FC(0.075) / persistence);
            case TU_DECAY_W: return expf(-dt * FC(0.14) / persistence);
            case TU_TAMB4: return powf(u[U_T_AMBIENT], 4.0f);
            case TU_MX: return m.x;
            case TU_MY: return m.y;
            case TU_MZ: return m.z;
            case TU_VMIX: return fx_clamp(dt * FC(0.32), 0.0f, FC(0.12));
            case TU_TMIX: return fx_clamp(dt * FC(0.18), 0.0f, FC(0.08));
            case TU_SMIX: return fx_clamp(dt * FC(0.12), 0.0f, FC(0.06));
            case TU_POWER: return firePower;
            case TU_POWER_ROOT: return powerRoot;
            case TU_THERMAL: return fx_min(powerRoot, 1.0f + FC(0.22) * (powerRoot - 1.0f));
            case TU_LIFT: return fx_clamp(u[U_LIFT], 0.0f, 4.0f);
            case TU_ENTRAIN: return fx_clamp(u[U_ENTRAIN], 0.0f, 3.0f);
            case TU_AMB_O2: return fx_max(u[U_OXYGEN], FC(0.001));
            case TU_HEAT: return 2150.0f + 1450.0f * u[U_HEAT_EFF];
            case TU_VORT_S: return FC(0.00135) * u[U_VORTICITY] * dt;
            case TU_TURB: return FC(0.075) + FC(0.16) * u[U_VORTICITY];
            case TU_BUOY: return fx_clamp(u[U_BUOYANCY], 0.0f, 4.0f);
            case TU_CINE: return fx_clamp(u[U_CINEMATIC], 0.0f, 1.0f);
            default: break;
        }
        if (i >= TU_SPRAY_X && i <= TU_SPRAY_Z) {  // spray momentum direction (shaders.ts:293-297)
            const float3 ext = fx_extent(u);
            const float ox = FC(0.035) * ext.x, oy = FC(0.50) * ext.y, oz = FC(0.5) * ext.z;
            const float tx = FC(0.52) * ext.x, ty = u[U_AIM_HEIGHT] * ext.y, tz = FC(0.5) * ext.z;
            const float dx = tx - ox, dy = ty - oy, dz = tz - oz;
            const float l = fx_length3(dx, dy, dz);
            return i == TU_SPRAY_X ? dx / l : (i == TU_SPRAY_Y ? dy / l : dz / l);
        }
        return 0.0f;
    }
    if (i < L.y) {
        const int k = (i - L.x) / X, x = (i - L.x) - k * X;
        const float nx = nrm(x, u[U_GRID_X]);
        if (k == TX_SWZ) return cosf(u[U_TIME] * FC(1.9) + nx * 25.0f);
        const FxBurnerGeom G = fx_burner_geom(u);
        const float px = nx * G.ext.x, ox = px - G.cx;
        if (k == TX_CELL) return sinf(px * 49.0f + time * FC(5.2));
        if (k == TX_LOBE) return sinf(ox / fx_max(G.radiusX, FC(0.001)) * FC(6.2) + time * FC(1.7));
        return ox * ox / (G.radiusX * G.radiusX);
    }
    if (i < L.z) {
        const int k = (i - L.y) / Y, y = (i - L.y) - k * Y;
        const float ny = nrm(y, u[U_GRID_Y]);
        if (k == TY_HE) return fx_smoothstep(FC(0.045), FC(0.15), ny) * (1.0f - fx_smoothstep(FC(0.80), 1.0f, ny));
        const float outflow = fx_smoothstep(FC(0.84), FC(0.995), ny);
        if (k == TY_OUT) return outflow;
        if (k == TY_DECAY) return expf(-outflow * dt * 15.0f / persistence);
        if (k == TY_MIX) return outflow * FC(0.16) / persistence;
        const FxBurnerGeom G = fx_burner_geom(u);
        const float oy = ny * G.ext.y - FC(0.075);
        return oy * oy / (FC(0.0022) * G.thickness * G.thickness);
    }
    if (i < L.ltx) {
        const int k = (i - L.z) / Z, z = (i - L.z) - k * Z;
        const float nz = nrm(z, u[U_GRID_Z]);
        if (k == TZ_SWX) return sinf(u[U_TIME] * FC(2.3) + nz * 22.0f);
        const FxBurnerGeom G = fx_burner_geom(u);
        const float pz = nz * G.ext.z, oz = pz - G.cz;
        if (k == TZ_CELL) return sinf(pz * 43.0f - time * FC(4.4));
        if (k == TZ_LOBE) return sinf(oz / fx_max(G.radiusZ, FC(0.001)) * FC(5.4) - time * FC(1.3));
        return oz * oz / (G.radiusZ * G.radiusZ);
    }
    if (i < L.lty) {  // turbulence x term, (y, z)
        const int j = i - L.ltx, z = j / Y, y = j - z * Y;
        const float ny = nrm(y, u[U_GRID_Y]), nz = nrm(z, u[U_GRID_Z]);
        return sinf(ny * 31.0f + nz * 19.0f + time * FC(3.1)) + FC(0.45) * sinf(ny * 67.0f - time * FC(5.3));
    }
    if (i < L.ltz) {  // turbulence y term, (x, z)
        const int j = i - L.lty, z = j / X, x = j - z * X;
        const float nx = nrm(x, u[U_GRID_X]), nz = nrm(z, u[U_GRID_Z]);
        return FC(0.12) * sinf(nx * 29.0f + nz * 23.0f - time * FC(4.1));
    }
    if (i < L.pulse) {  // turbulence z term, (x, y)
        const int j = i - L.ltz, y = j / X, x = j - y * X;
        const float nx = nrm(x, u[U_GRID_X]), ny = nrm(y, u[U_GRID_Y]);
        return cosf(ny * 27.0f - nx * 21.0f + time * FC(2.7)) + FC(0.45) * cosf(ny * 59.0f + time * FC(4.7));
    }
    {  // burner pulse, (x, z)
        const int j = i - L.pulse, z = j / X, x = j - z * X;
        const FxBurnerGeom G = fx_burner_geom(u);
        const float px = nrm(x, u[U_GRID_X]) * G.ext.x, pz = nrm(z, u[U_GRID_Z]) * G.ext.z;
        return FC(0.84) + FC(0.16) * sinf(time * FC(3.7) + px * 27.0f + pz * 21.0f);
    }
}

struct FxCellOut {
    float4 flow;
    float4 species;
    float reaction;
};

// simulate (shaders.ts:151-342) for cell (x, y, z): advection, diffusion, source,
// boundary ambient, liquid cooling, entrainment, Arrhenius burn, vorticity confinement,
// turbulence, buoyancy, spray momentum, radiation, open-top outflow and wall clamps.
// P, ut (the per-step table's uniform entries, TU_*) and dc are the same for every cell of a
// simulation: the source pass stages them in shared memory; tab (the per-coordinate tables)
// and the fields come from global memory.
template <bool EARLY, class Acc>
FXD FxCellOut fx_simulate_cell(const FxParams& P, const FxGrid& g, int x, int y, int z, const Acc& a,
                               const float* __restrict__ tab, const float* ut, const FxDivc* dc) {
    const float* u = P.u;
    const int X = g.X, Y = g.Y, Z = g.Z;
    const FxTabLayout L = fx_tab_layout(X, Y, Z);
    const int id = x + X * (y + Y * z);
    float picx = (float)x + 0.5f, picy = (float)y + 0.5f, picz = (float)z + 0.5f;
    float dt = u[U_DT];

    float4 orig = a.flow(id);
    const float3 metric = make_float3(ut[TU_MX], ut[TU_MY], ut[TU_MZ]);

    // The neighbour terms: the 6-neighbour averages of the diffusion and the curl and normalised
    // temperature gradient of the vorticity confinement, each the reference's expression. EARLY
    // evaluates them before the advection, so that only these values, not the 12 neighbour
    // records, stay live through the update and the neighbour loads overlap the advection's
    // dependent loads (faster up to about 10 M cells: HD 0.185 against 0.194 ms per pass,
    // 192x288x192 0.604 against 0.618); otherwise they are evaluated where the reference does
    // (256^3: 0.964 against 1.010 ms). The results are the same either way.
    // 6 neighbours with clamped (Neumann) addressing (shaders.ts:43-51)
    const int oL = x > 0 ? id - 1 : id, oR = x < X - 1 ? id + 1 : id;
    const int oB = y > 0 ? id - X : id, oT = y < Y - 1 ? id + X : id;
    const int oK = z > 0 ? id - X * Y : id, oF = z < Z - 1 ? id + X * Y : id;
    float vax, vay, vaz, ta;  // shaders.ts:177-180
    float cx, cy, cz;         // curl (shaders.ts:258-263)
    float gx, gy, gz;         // normalised grad(T) (shaders.ts:264-268)
    float4 avg;               // species diffusion (shaders.ts:182-187)
    float4 left, right, bottom, top, back, front;
    if constexpr (EARLY) {
        const float4 l = a.flow(oL), r = a.flow(oR), bo = a.flow(oB), t = a.flow(oT), k = a.flow(oK), f = a.flow(oF);
        vax = fx_divc(l.x + r.x + bo.x + t.x + k.x + f.x, dc[DIVC_SIX]);
        vay = fx_divc(l.y + r.y + bo.y + t.y + k.y + f.y, dc[DIVC_SIX]);
        vaz = fx_divc(l.z + r.z + bo.z + t.z + k.z + f.z, dc[DIVC_SIX]);
        ta = fx_divc(l.w + r.w + bo.w + t.w + k.w + f.w, dc[DIVC_SIX]);
        cx = 0.5f * ((t.z - bo.z) * metric.y - (f.y - k.y) * metric.z);
        cy = 0.5f * ((f.x - k.x) * metric.z - (r.z - l.z) * metric.x);
        cz = 0.5f * ((r.y - l.y) * metric.x - (t.x - bo.x) * metric.y);
        gx = 0.5f * ((r.w - l.w) * metric.x) + FC(0.00001);
        gy = 0.5f * ((t.w - bo.w) * metric.y) + FC(0.00001);
        gz = 0.5f * ((f.w - k.w) * metric.z) + FC(0.00001);
        const float gl = fx_length3(gx, gy, gz);
        gx = gx / gl;
        gy = gy / gl;
        gz = gz / gl;
        const float4 sl = a.species(oL), sr = a.species(oR);
        const float4 sb = a.species(oB), st = a.species(oT);
        const float4 sk = a.species(oK), sf = a.species(oF);
        avg = make_float4(fx_divc(sl.x + sr.x + sb.x + st.x + sk.x + sf.x, dc[DIVC_SIX]),
                          fx_divc(sl.y + sr.y + sb.y + st.y + sk.y + sf.y, dc[DIVC_SIX]),
                          fx_divc(sl.z + sr.z + sb.z + st.z + sk.z + sf.z, dc[DIVC_SIX]),
                          fx_divc(sl.w + sr.w + sb.w + st.w + sk.w + sf.w, dc[DIVC_SIX]));
    }

    float btx = picx - orig.x * dt * metric.x;
    float bty = picy - orig.y * dt * metric.y;
    float btz = picz - orig.z * dt * metric.z;
    const FxTri tri = fx_tri_setup(g, u, btx, bty, btz);
    float4 flow = fx_trilinear(g, tri, [&](int i) { return a.flow(i); });
    float4 species = fx_trilinear(g, tri, [&](int i) { return a.species(i); });
    species = make_float4(fx_max(species.x, 0.0f), fx_max(species.y, 0.0f), fx_max(species.z, 0.0f),
                          fx_max(species.w, 0.0f));

    if constexpr (!EARLY) {
        left = a.flow(oL);
        right = a.flow(oR);
        bottom = a.flow(oB);
        top = a.flow(oT);
        back = a.flow(oK);
        front = a.flow(oF);
    }
    {  // 6-neighbour diffusion of velocity and temperature (shaders.ts:177-180)
        if constexpr (!EARLY) {
            vax = fx_divc(left.x + right.x + bottom.x + top.x + back.x + front.x, dc[DIVC_SIX]);
            vay = fx_divc(left.y + right.y + bottom.y + top.y + back.y + front.y, dc[DIVC_SIX]);
            vaz = fx_divc(left.z + right.z + bottom.z + top.z + back.z + front.z, dc[DIVC_SIX]);
        }
        float vm = ut[TU_VMIX];
        flow.x = fx_mix(flow.x, vax, vm);
        flow.y = fx_mix(flow.y, vay, vm);
        flow.z = fx_mix(flow.z, vaz, vm);
        if constexpr (!EARLY) ta = fx_divc(left.w + right.w + bottom.w + top.w + back.w + front.w, dc[DIVC_SIX]);
        flow.w = fx_mix(flow.w, ta, ut[TU_TMIX]);
    }
    {  // species diffusion (shaders.ts:182-187)
        if constexpr (!EARLY) {
            float4 sl = a.species(oL), sr = a.species(oR);
            float4 sb = a.species(oB), st = a.species(oT);
            float4 sk = a.species(oK), sf = a.species(oF);
            avg = make_float4(fx_divc(sl.x + sr.x + sb.x + st.x + sk.x + sf.x, dc[DIVC_SIX]),
                              fx_divc(sl.y + sr.y + sb.y + st.y + sk.y + sf.y, dc[DIVC_SIX]),
                              fx_divc(sl.z + sr.z + sb.z + st.z + sk.z + sf.z, dc[DIVC_SIX]),
                              fx_divc(sl.w + sr.w + sb.w + st.w + sk.w + sf.w, dc[DIVC_SIX]));
        }
        species = fx_mix4(species, avg, ut[TU_SMIX]);
    }

    // Source injection (shaders.ts:189-201); the sphere list replaces the burner.
    const float firePower = ut[TU_POWER];
    const float powerRoot = ut[TU_POWER_ROOT];
    const float thermalPower = ut[TU_THERMAL];
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
    } else {  // emitter (shaders.ts:101-133) from the per-step tables
        const float radial = __ldg(tab + L.x + TX_RAD * X + x) + __ldg(tab + L.z + TZ_RAD * Z + z);
        const float vertical = __ldg(tab + L.y + TY_VERT * Y + y);
        const float cellular = FC(0.76) + FC(0.24) * __ldg(tab + L.x + TX_CELL * X + x) * __ldg(tab + L.z + TZ_CELL * Z + z);
        const float lobeArg = __ldg(tab + L.x + TX_LOBE * X + x) * __ldg(tab + L.z + TZ_LOBE * Z + z);
        const float lobes = fx_mix(FC(0.48), FC(1.18), fx_smoothstep_c(FC(-0.42), lobeArg, dc[DIVC_LOBE]));
        const float texture = fx_mix(cellular, cellular * lobes, ut[TU_CINE]);
        const float pulse = __ldg(tab + L.pulse + z * X + x);
        source = expf(-(radial + vertical)) * texture * pulse;
        species.x = fx_max(species.x, source * u[U_FUEL_RATE] * firePower);
        flow.w = fx_max(flow.w, u[U_T_AMBIENT] + source * 1180.0f * thermalPower);
    }
    {
        float swx = __ldg(tab + L.z + TZ_SWX * Z + z);
        float swy = 0.0f;
        float swz = __ldg(tab + L.x + TX_SWZ * X + x);
        float s = source * dt * FC(0.11) * u[U_VORTICITY] * powerRoot;
        flow.x = flow.x + swx * s;
        flow.y = flow.y + swy * s;
        flow.z = flow.z + swz * s;
        flow.y += source * dt * FC(0.52) * ut[TU_LIFT] * powerRoot;
    }

    if (x == 0 || x == X - 1 || z == 0 || z == Z - 1 || y == Y - 1) {  // shaders.ts:203-208
        species.y = fx_max(species.y, u[U_OXYGEN]);
        flow.w = fx_mix(flow.w, u[U_T_AMBIENT], FC(0.035));
    }

    // Liquid cooling and vapor (shaders.ts:212-215). With no liquid (water == +0) every
    // product below is +0 and the updates reduce exactly to max/clamp of the inputs.
    const uint32_t liquidRaw = a.liquid(id);
    float water = fx_clamp((float)liquidRaw * (1.0f / 4096.0f) * FC(3.4), 0.0f, 5.0f);
    if (liquidRaw) {
        float evaporation = water * fx_smoothstep_c(335.0f, flow.w, dc[DIVC_EVAP]) * dt * FC(13.5);
        flow.w = fx_max(u[U_T_AMBIENT], flow.w - evaporation * 2080.0f - water * dt * 260.0f);
        species.w = fx_clamp(species.w + evaporation * FC(2.15), 0.0f, 3.0f);
    } else {
        flow.w = fx_max(u[U_T_AMBIENT], flow.w);             // x - (+0) == x exactly
        species.w = fx_clamp(species.w + 0.0f, 0.0f, 3.0f);  // x + (+0) maps -0 to +0, as the full form
    }

    // O2 entrainment (shaders.ts:220-232)
    const float entrainment = ut[TU_ENTRAIN];
    const float ambientOxygen = ut[TU_AMB_O2];
    float oxygenDeficit = fx_clamp(fx_divc(ambientOxygen - species.y, dc[DIVC_AMBIENT_O2]), 0.0f, 1.0f);
    float fuelCore = fx_smoothstep_c(FC(0.30), species.x, dc[DIVC_FUELCORE]);
    float interfaceWeight = oxygenDeficit * fx_mix(1.0f, FC(0.18), fuelCore);
    float entrainmentMix = fx_clamp(dt * entrainment *
                                        (FC(0.12) + FC(0.28) * fx_length3(flow.x, flow.y, flow.z) +
                                         FC(0.22) * fx_smoothstep_c(400.0f, flow.w, dc[DIVC_ENTRAIN_T])) *
                                        interfaceWeight,
                                    0.0f, FC(0.08));
    species.y = fx_mix(species.y, ambientOxygen, entrainmentMix);

    // Arrhenius burn bounded by the 1:4 fuel:O2 ratio (shaders.ts:234-256)
    float fuelBefore = fx_max(species.x, 0.0f);
    float oxygenBefore = fx_max(species.y, 0.0f);
    float availableFuel = fx_min(fuelBefore, oxygenBefore * FC(0.25));
    float ignition = fx_smoothstep_c(690.0f, flow.w, dc[DIVC_IGNITION]);
    // 1 - exp(-arrhenius * ignition * dt). Below ignition (ignition == +0) the exponent is
    // -0 for any finite rate (the rate is clamped to [0, 80]) and the factor is exactly
    // +0, so the rate need not be evaluated; with no liquid exp(-water * 18) is exactly 1.
    float growth = 0.0f;
    if (!(ignition == 0.0f)) {
        float safeFuel = fx_max(fuelBefore, FC(0.00001));
        float safeOxygen = fx_max(oxygenBefore, FC(0.00001));
        float activation = expf(-15000.0f / fx_max(flow.w, u[U_T_AMBIENT]));
        float arrhenius =
            fx_clamp(FC(2.5e6) * activation * powf(safeFuel, FC(-0.30)) * powf(safeOxygen, FC(1.30)), 0.0f, 80.0f);
        growth = 1.0f - expf(-arrhenius * ignition * dt);
    }
    float requestedBurn = availableFuel * growth;
    if (liquidRaw) requestedBurn = requestedBurn * expf(-water * 18.0f);
    float burn = fx_clamp(requestedBurn, 0.0f, availableFuel);
    float richness = fx_clamp(1.0f - oxygenBefore / fx_max(fuelBefore * 4.0f, FC(0.00001)), 0.0f, 1.0f);
    species.x = fx_max(0.0f, fuelBefore - burn);
    species.y = fx_max(0.0f, oxygenBefore - burn * 4.0f);
    species.z = fx_clamp(species.z + burn * (1.0f + richness * FC(1.8)), 0.0f, 3.0f);
    species.w = fx_clamp(species.w + burn * FC(0.62), 0.0f, 3.0f);
    flow.w += burn * ut[TU_HEAT];
    float reaction = fx_clamp(fx_divc(burn, dc[DIVC_DT]) * FC(0.22), 0.0f, 4.0f);

    {  // vorticity confinement: curl x grad(T) (shaders.ts:258-272)
        if constexpr (!EARLY) {
            cx = 0.5f * ((top.z - bottom.z) * metric.y - (front.y - back.y) * metric.z);
            cy = 0.5f * ((front.x - back.x) * metric.z - (right.z - left.z) * metric.x);
            cz = 0.5f * ((right.y - left.y) * metric.x - (top.x - bottom.x) * metric.y);
            gx = 0.5f * ((right.w - left.w) * metric.x) + FC(0.00001);
            gy = 0.5f * ((top.w - bottom.w) * metric.y) + FC(0.00001);
            gz = 0.5f * ((front.w - back.w) * metric.z) + FC(0.00001);
            float gl = fx_length3(gx, gy, gz);
            gx = gx / gl;
            gy = gy / gl;
            gz = gz / gl;
        }
        const float vs = ut[TU_VORT_S];
        flow.x = flow.x + (gy * cz - gz * cy) * vs;
        flow.y = flow.y + (gz * cx - gx * cz) * vs;
        flow.z = flow.z + (gx * cy - gy * cx) * vs;
    }
    {  // height-enveloped turbulence (shaders.ts:274-285)
        float hotPlume = fx_smoothstep_c(520.0f, flow.w, dc[DIVC_HOTPLUME]);
        float heightEnvelope = __ldg(tab + L.y + TY_HE * Y + y);
        float ltx = __ldg(tab + L.ltx + z * Y + y);
        float lty = __ldg(tab + L.lty + z * X + x);
        float ltz = __ldg(tab + L.ltz + y * X + x);
        float ts = ut[TU_TURB] * hotPlume * heightEnvelope * dt;
        flow.x = flow.x + ltx * ts;
        flow.y = flow.y + lty * ts;
        flow.z = flow.z + ltz * ts;
    }
    {  // buoyancy (shaders.ts:287-288)
        float buoyancy = fx_clamp(fx_divc(flow.w - u[U_T_AMBIENT], dc[DIVC_BUOYANCY]), FC(-0.1), FC(1.2));
        flow.y += buoyancy * dt * FC(0.72) * ut[TU_BUOY];
    }
    if (liquidRaw) species.z *= expf(-water * dt * FC(4.8));  // exp(-0) == 1 exactly otherwise
    {  // spray momentum (shaders.ts:293-297)
        const float dx = ut[TU_SPRAY_X], dy = ut[TU_SPRAY_Y], dz = ut[TU_SPRAY_Z];
        flow.x = flow.x + dx * water * dt * FC(0.82);
        flow.y = flow.y + dy * water * dt * FC(0.82);
        flow.z = flow.z + dz * water * dt * FC(0.82);
    }
    // radiation and decay (shaders.ts:299-304); the decay factors come from the table
    // pow(T, 4): cells at exactly the ambient temperature (every cold cell clamped to it
    // above) take the per-step table value, which is the same powf of the same input
    const float tRad = fx_max(flow.w, 0.0f);
    const float tamb4 = ut[TU_TAMB4];
    const float t4 = tRad == u[U_T_AMBIENT] ? tamb4 : powf(tRad, 4.0f);
    float radiation = fx_divc(FC(5.67e-8) * (tamb4 - t4), dc[DIVC_RADIATION]);
    flow.w = fx_max(u[U_T_AMBIENT], flow.w + dt * radiation);
    species.z *= ut[TU_DECAY_Z];
    species.w *= ut[TU_DECAY_W];

    // open-top outflow (shaders.ts:308-321)
    float outflow = __ldg(tab + L.y + TY_OUT * Y + y);
    species.x *= 1.0f - outflow;
    float outflowDecay = __ldg(tab + L.y + TY_DECAY * Y + y);
    species.z *= outflowDecay;
    species.w *= outflowDecay;
    flow.w = fx_mix(flow.w, u[U_T_AMBIENT], __ldg(tab + L.y + TY_MIX * Y + y));
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
// Jacobi constants as pairs, for fx_jacobi4.
struct FxJacobiConst2 {
    fx_f2 rcp, negDenom;
    float wxS, wyS, wzS, denom, rcpS;
    bool fast;
};
FXD FxJacobiConst2 fx_jacobi_const2(const FxJacobiConst& c, float rcp, bool fast) {
    return FxJacobiConst2{fx_pack2(rcp, rcp), fx_pack2(-c.denom, -c.denom), c.wx, c.wy, c.wz, c.denom, rcp, fast};
}

// The end of fx_jacobi4 from the six weighted pair sums: the numerators and the division.
template <bool INLINE_RARE>
FXD float4 fx_jacobi4_finish(const FxJacobiConst2& c, fx_f2 x01, fx_f2 x23, fx_f2 y01, fx_f2 y23, fx_f2 z01, fx_f2 z23,
                             float4 d) {
    const fx_f2 n01 = fx_sub2(fx_add2(fx_add2(x01, y01), z01), fx_pack2(d.x, d.y));
    const fx_f2 n23 = fx_sub2(fx_add2(fx_add2(x23, y23), z23), fx_pack2(d.z, d.w));
    const float2 a = fx_unpack2(n01), b = fx_unpack2(n23);
    if (!c.fast) return make_float4(__fdiv_rn(a.x, c.denom), __fdiv_rn(a.y, c.denom), __fdiv_rn(b.x, c.denom), __fdiv_rn(b.y, c.denom));
    // Markstein's step on both pairs: q = x rcp, e = fma(q, -d, x) = x - q d, q + e rcp
    const fx_f2 q01 = fx_mul2(n01, c.rcp), q23 = fx_mul2(n23, c.rcp);
    const fx_f2 r01 = fx_fma2(fx_fma2(q01, c.negDenom, n01), c.rcp, q01);
    const fx_f2 r23 = fx_fma2(fx_fma2(q23, c.negDenom, n23), c.rcp, q23);
    const float2 ra = fx_unpack2(r01), rb = fx_unpack2(r23);
    // every |x| inside [2^-96, FLT_MAX]? (false for zeros, tiny x, infinities and NaN)
    const float lo = 1.2621774483536189e-29f, hi = 3.402823466e38f;
    const bool ok = (fabsf(a.x) >= lo) & (fabsf(a.x) <= hi) & (fabsf(a.y) >= lo) & (fabsf(a.y) <= hi) &
                    (fabsf(b.x) >= lo) & (fabsf(b.x) <= hi) & (fabsf(b.y) >= lo) & (fabsf(b.y) <= hi);
    if (ok) return make_float4(ra.x, ra.y, rb.x, rb.y);
    if (INLINE_RARE) {  // zeros keep their sign; infinities and NaN pass through, as fx_div_rare
        auto ieee = [&](float x) { return (x == 0.0f || !(fabsf(x) <= hi)) ? x : __fdiv_rn(x, c.denom); };
        return make_float4(ieee(a.x), ieee(a.y), ieee(b.x), ieee(b.y));
    }
    return make_float4(fx_div_by_const(a.x, c.denom, c.rcpS), fx_div_by_const(a.y, c.denom, c.rcpS),
                       fx_div_by_const(b.x, c.denom, c.rcpS), fx_div_by_const(b.y, c.denom, c.rcpS));
}

// Four consecutive x cells of one Jacobi sweep (the operations of fx_jacobi_numerator and
// fx_div_by_const, cell by cell, two cells per instruction): pc holds the cells, l and r
// their outer x neighbours, pb/pt/pk/pf the y-1, y+1, z-1, z+1 rows, d the divergence.
// A group with a numerator outside the checked range takes the IEEE division for its four
// cells (the same quotients: inside the range the checked path equals it), through the
// out-of-line rare path of fx_div_by_const, or inline (INLINE_RARE: no call in the caller's
// loop; measured faster in the resident kernel at HD, 5.60 against 6.02 us per sweep, and
// 1 % slower in the two-sweep kernel at 508^3).
// A packed multiply feeding a packed add is contracted into a packed fma by the code
// generator (measured on B200), which rounds once instead of twice, so the weight products
// are either scalar multiplies (never contracted) or, with PACKED_W, packed fused
// multiply-adds of -0: RN(w s + -0) = RN(w s) for every w and s, zeros' signs included, and
// an fma feeding an add is not contracted. The -0 is computed from the run-time divisor
// (finite), so the fma cannot be folded back into a multiply. PACKED_W measured 5.61
// against 5.65 us per sweep in the resident kernel with the copy warp at HD, and 1 % slower
// per step in the two-sweep kernel at 508^3.
template <bool INLINE_RARE = false, bool PACKED_W = false>
FXD float4 fx_jacobi4(const FxJacobiConst2& c, float l, float4 pc, float r, float4 pb, float4 pt, float4 pk, float4 pf,
                      float4 d) {
    const fx_f2 mid = fx_pack2(pc.y, pc.z);
    const fx_f2 lr01 = fx_add2(fx_pack2(l, pc.x), mid);
    const fx_f2 lr23 = fx_add2(mid, fx_pack2(pc.w, r));
    const fx_f2 bt01 = fx_add2(fx_pack2(pb.x, pb.y), fx_pack2(pt.x, pt.y));
    const fx_f2 bt23 = fx_add2(fx_pack2(pb.z, pb.w), fx_pack2(pt.z, pt.w));
    const fx_f2 kf01 = fx_add2(fx_pack2(pk.x, pk.y), fx_pack2(pf.x, pf.y));
    const fx_f2 kf23 = fx_add2(fx_pack2(pk.z, pk.w), fx_pack2(pf.z, pf.w));
    if constexpr (PACKED_W) {
        const float nzs = -0.0f * fabsf(c.denom);
        const fx_f2 nz = fx_pack2(nzs, nzs);
        const fx_f2 wx2 = fx_pack2(c.wxS, c.wxS), wy2 = fx_pack2(c.wyS, c.wyS), wz2 = fx_pack2(c.wzS, c.wzS);
        return fx_jacobi4_finish<INLINE_RARE>(c, fx_fma2(wx2, lr01, nz), fx_fma2(wx2, lr23, nz), fx_fma2(wy2, bt01, nz),
                                              fx_fma2(wy2, bt23, nz), fx_fma2(wz2, kf01, nz), fx_fma2(wz2, kf23, nz), d);
    } else {
        const float2 s01 = fx_unpack2(lr01), s23 = fx_unpack2(lr23), u01 = fx_unpack2(bt01), u23 = fx_unpack2(bt23);
        const float2 v01 = fx_unpack2(kf01), v23 = fx_unpack2(kf23);
        const fx_f2 x01 = fx_pack2(__fmul_rn(c.wxS, s01.x), __fmul_rn(c.wxS, s01.y));
        const fx_f2 x23 = fx_pack2(__fmul_rn(c.wxS, s23.x), __fmul_rn(c.wxS, s23.y));
        const fx_f2 y01 = fx_pack2(__fmul_rn(c.wyS, u01.x), __fmul_rn(c.wyS, u01.y));
        const fx_f2 y23 = fx_pack2(__fmul_rn(c.wyS, u23.x), __fmul_rn(c.wyS, u23.y));
        const fx_f2 z01 = fx_pack2(__fmul_rn(c.wzS, v01.x), __fmul_rn(c.wzS, v01.y));
        const fx_f2 z23 = fx_pack2(__fmul_rn(c.wzS, v23.x), __fmul_rn(c.wzS, v23.y));
        return fx_jacobi4_finish<INLINE_RARE>(c, x01, x23, y01, y23, z01, z23, d);
    }
}

// One cell of fx_jacobi4 (the same numerator; the checked constant division when enabled).
FXD float fx_jacobi1(const FxJacobiConst2& c, float l, float r, float b, float t, float k, float f, float div) {
    const float n = fx_jacobi_numerator(FxJacobiConst{c.wxS, c.wyS, c.wzS, c.denom}, l, r, b, t, k, f, div);
    return c.fast ? fx_div_by_const(n, c.denom, c.rcpS) : __fdiv_rn(n, c.denom);
}

