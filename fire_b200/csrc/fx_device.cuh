// fx_device.cuh — device-side building blocks shared by the Fire-X kernels.
//
// The WGSL builtins are written from their WGSL-spec definitions so the f32 kernels
// evaluate every reference expression as the same sequence of IEEE operations:
//   max(a,b) = (a < b) ? b : a          min(a,b) = (b < a) ? b : a
//   clamp(x,lo,hi) = min(max(x,lo),hi)  mix(a,b,t) = a*(1-t) + b*t
//   smoothstep(e0,e1,x) = t*t*(3-2t), t = clamp((x-e0)/(e1-e0), 0, 1)
// Files that include this header for the reference-faithful path are compiled with
// --fmad=false (no contraction into fused multiply-add).
#pragma once

#include <cuda.h>  // CUtensorMap

#include <cstdint>
#include <cuda_fp16.h>

#include "../../include/firex.h"

// Constant divisors of simulate. Each slot holds d > 0, rcp = RN(1/d) and the range
// [lo, hi] of |x| where Markstein's correction step (fx_div_checked) reproduces IEEE
// x / d; ok = 1 once the engine has checked that on the device for every float x.
struct __align__(16) FxDivc {  // one 16-byte load brings d, rcp, lo and hi
    float d, rcp, lo, hi;         // lo = +inf when the checked path is not enabled
    int ok, pad[3];               // host record of the device check
};
enum FxDivSlot {
    DIVC_SIX = 0,        // the 6-neighbour averages (shaders.ts:177-186)
    DIVC_FUELCORE,       // smoothstep(0.30, 0.78, fuel)
    DIVC_ENTRAIN_T,      // smoothstep(400, 1500, T)
    DIVC_IGNITION,       // smoothstep(690, 930, T)
    DIVC_HOTPLUME,       // smoothstep(520, 1650, T)
    DIVC_EVAP,           // smoothstep(335, 1040, T)
    DIVC_LOBE,           // smoothstep(-0.42, 0.48, lobe)
    DIVC_BUOYANCY,       // (T - T_amb) / 1500
    DIVC_AMBIENT_O2,     // (ambientOxygen - O2) / ambientOxygen
    DIVC_DT,             // burn / max(dt, 0.0001)
    DIVC_RADIATION,      // ... / (1005 * persistence)
    DIVC_COUNT
};

// Per-step parameter block: the reference's 44-float uniform block (shaders.ts:2-14,
// written by FireXEngine.writeUniforms, FireXEngine.ts:2043-2113) followed by the
// sphere-emitter extension.
struct FxParams {
    float u[FIREX_UNIFORM_FLOATS];
    int32_t emitter_mode;
    float jitter;
    int32_t num_spheres;
    int32_t pad;
    firex_sphere spheres[FIREX_MAX_SPHERES];
};

// Uniform slots (vec4 members of Parameters, shaders.ts:2-14).
enum FxSlot {
    U_GRID_X = 0, U_GRID_Y = 1, U_GRID_Z = 2,
    U_DT = 4, U_TIME = 5,
    U_FUEL_RATE = 8, U_OXYGEN = 9, U_HEAT_EFF = 10, U_VORTICITY = 11,
    U_T_AMBIENT = 15,
    U_VIEW_MODE = 24, U_AIM_HEIGHT = 25,
    U_BURNER_X = 28, U_BURNER_Z = 29, U_THICKNESS = 30, U_FIRE_POWER = 31,
    U_DOMAIN_X = 32, U_DOMAIN_Y = 33, U_DOMAIN_Z = 34,
    U_LIFT = 36, U_BUOYANCY = 37, U_PERSISTENCE = 38,
    U_ENTRAIN = 40, U_CINEMATIC = 42,
};

#define FXD __device__ __forceinline__

FXD float fx_max(float a, float b) { return (a < b) ? b : a; }
FXD float fx_min(float a, float b) { return (b < a) ? b : a; }
FXD float fx_clamp(float x, float lo, float hi) { return fx_min(fx_max(x, lo), hi); }
FXD float fx_mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
FXD float fx_smoothstep(float e0, float e1, float x) {
    float t = fx_clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
FXD float4 fx_mix4(float4 a, float4 b, float t) {
    return make_float4(fx_mix(a.x, b.x, t), fx_mix(a.y, b.y, t), fx_mix(a.z, b.z, t), fx_mix(a.w, b.w, t));
}
FXD float fx_length3(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

// Float constant rounded from its double literal, as WGSL concretises abstract floats.
#define FC(v) (static_cast<float>(v))

// Grids hold fewer than 2^31 cells, so 32-bit cell offsets are exact.
struct FxGrid {
    int X, Y, Z;
    __device__ __forceinline__ int idx(int x, int y, int z) const {
        x = x < 0 ? 0 : (x > X - 1 ? X - 1 : x);
        y = y < 0 ? 0 : (y > Y - 1 ? Y - 1 : y);
        z = z < 0 ? 0 : (z > Z - 1 ? Z - 1 : z);
        return x + X * (y + Y * z);
    }
};

// domainExtent() and cellMetric() (shaders.ts:35-41).
FXD float3 fx_extent(const float* u) {
    return make_float3(fx_max(u[U_DOMAIN_X], 0.001f), fx_max(u[U_DOMAIN_Y], 0.001f), fx_max(u[U_DOMAIN_Z], 0.001f));
}
FXD float3 fx_metric(const float* u) {
    float3 e = fx_extent(u);
    return make_float3(u[U_GRID_X] / e.x, u[U_GRID_Y] / e.y, u[U_GRID_Z] / e.z);
}

// Sphere emitter mask (extension): |c + 0.5 - center|^2 <= r^2, float, fixed order.
// Written with explicit round-to-nearest intrinsics so the integer mask is the same in
// every translation unit, whatever its contraction flags.
FXD bool fx_sphere_inside(const firex_sphere& s, int x, int y, int z) {
    float dx = __fsub_rn(__fadd_rn((float)x, 0.5f), s.center[0]);
    float dy = __fsub_rn(__fadd_rn((float)y, 0.5f), s.center[1]);
    float dz = __fsub_rn(__fadd_rn((float)z, 0.5f), s.center[2]);
    float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    return d2 <= __fmul_rn(s.radius, s.radius);
}

// splitmix64 (Steele, Lea, Flood 2014) for the seeded initial velocity noise.
FXD uint64_t fx_splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Seeded initial velocity noise (extension): component comp of cell id, uniform in
// [-a, a] from 24 random bits.
FXD float fx_velocity_noise(uint64_t seed, uint64_t cell, int comp, float a) {
    uint64_t h = fx_splitmix64(fx_splitmix64(seed ^ 0x6A09E667F3BCC909ull) + cell * 4u + (uint64_t)comp);
    float u = __fmul_rn((float)(h >> 40), 1.0f / 16777216.0f);
    return __fmul_rn(a, __fsub_rn(__fmul_rn(2.0f, u), 1.0f));
}

// ---------------------------------------------------------------------------------------
// Device-resident simulation descriptor. Parities and counters live on the device and
// are advanced by the step epilogue kernel, so a whole step (or a batch of simulations
// stepping together) is a fixed sequence of launches that a CUDA graph can replay with
// no per-step host arguments. The host keeps a mirror of the same counters, advanced
// by the same rules, for reads between steps.
enum FxStorage { FX_STORAGE_F32 = 0, FX_STORAGE_MIXED = 1 };

struct __align__(16) FxSimDev {
    FxParams prm;          // parameters of the running step (time fields set by step_begin)
    int X, Y, Z;
    int P, R;              // primary / residual Jacobi sweeps per step
    int mode;              // FIREX_PRESSURE_WARM_F32 / _F16 / _COLD_F32 (resolved)
    int storage;           // FxStorage
    int active;            // 0: skipped by every kernel (batch slot parked)
    int fi, si, pi;        // flow, species, pressure parity at the start of the step
    int pad0;
    double simTime;        // FireXEngine.simulationTime
    double dt;             // dt of the next step
    long long frame;       // FireXEngine.frameIndex
    uint64_t seed;
    float jitterAmp;
    int pad1;
    float metric[4];       // grid / domainExtent (shaders.ts:39-41), host-computed in f32
    float jc[4];           // Jacobi wx, wy, wz, 2(wx+wy+wz) (shaders.ts:386-389), f32
    float jcRcp;           // RN(1 / jc[3])
    int jcFastDiv;         // 1: x / jc[3] may use fx_div_by_const (checked exhaustively)
    int pad2[2];
    void* flow[2];         // float4 records (both storages)
    void* species[2];      // float4 (F32) or 4 x half (MIXED)
    void* p[2];            // primary pressure: float (F32 / COLD) or half (F16 / MIXED)
    void* corr[2];         // residual pressure (aliases p[] in branch C)
    float* div;
    float* reaction;
    uint32_t* liquid;
    float* tab;            // per-step tables of simulate (fx_step_math.cuh)
    FxDivc divc[DIVC_COUNT];
    float4* part[2];       // droplets (2 float4 each: position + age, velocity + mass), ping-pong
    float4* pdens;         // droplet density, near density, pressure, near pressure
    int np;                // droplet count
    int pti;               // droplets of the current state: part[pti]
    int water;             // 1: the particle passes run in this step (waterEnabled, waterFlow > 0.001)
    int waterPad;
    uint2* render[3];      // render volumes (4 x FP16 per cell): flow, chemistry, media
    int renderPack;        // 1: the step ends by packing the render volumes
    int renderPad;
    unsigned* sync;        // [2]: error word (a bounded device wait expired); from
                           // FX_RES_FLAGS: the resident Jacobi's per-box flags of both
                           // phases (zeroed at every step start)
    int tmapOk;            // 1: tmap holds valid tensor maps (FP32 pressure)
    int tmapPad[15];
    CUtensorMap tmap[5];   // pressure pair, correction pair, divergence (fx_jacobi_zm2t.cuh)
};

// Work decomposition shared by every batched pass: each pass walks a flat list of
// bricks across all simulations of a batch; start[shape][s] is the first brick of
// simulation s (prefix sums over the batch), so one launch covers uneven grids.
#define FX_MAX_BATCH 512
enum FxShape {
    FX_SHAPE_CELL = 0,
    FX_SHAPE_ROW4 = 1,
    FX_SHAPE_COL = 2,
    FX_SHAPE_ZM = 3,
    FX_SHAPE_TAB = 4,
    FX_SHAPE_RES = 5,  // one CTA per box of the resident Jacobi (fx_jacobi_res.cuh)
    FX_SHAPE_PART = 6, // FX_SPH_DROPLETS droplets per brick (members whose water runs)
    FX_NSHAPES = 7
};

// Box decomposition of one simulation for the resident Jacobi: boxes of by x bz rows of
// full x rows, nby x nbz of them (CTA b owns box (b % nby, b / nby)).
struct FxResBox {
    int by, bz, nby, nbz;
};
// CELL: 32 x BY x (8 / BY) cells, one thread per cell (simulate); BY = FX_CELL_BY unless
//       the plan tunes it (firex_set_tiles).
// ROW4: 256 groups of 4 consecutive x cells in memory order (stencils).
// COL : tiles x z chunks of the two-sweep Jacobi pass (see fx_jacobi_zm2.cuh).
// ZM  : z-marching tiles of the single-sweep Jacobi (see fx_jacobi_zm.cuh).
// TAB : 256 entries of the per-step tables of simulate.
#define FX_CELL_BX 32
#define FX_CELL_BY 4
#define FX_ROW4_THREADS 256
#define FX_SPH_THREADS 256                    // threads of the droplet passes: one warp per droplet
#define FX_SPH_DROPLETS (FX_SPH_THREADS / 32)  // droplets per brick

struct FxBatchDev {
    int nsims;
    int pad;
    int total[FX_NSHAPES];
    int colTileX, colTileY;        // interior tile of the COL shape
    FxSimDev* sims[FX_MAX_BATCH];
    int start[FX_NSHAPES][FX_MAX_BATCH + 1];
    FxResBox res[FX_MAX_BATCH];
};

// Buffers of launch `launch` of a solve phase: launches alternate between the two
// buffers of the phase starting from the warm-start parity (primary, branches A and B)
// or from buffer 0 (residual, and the cold primary of branch C); the first launch of a
// cleared solve has a zero input.
struct FxSolveBufs {
    const void* pin;
    void* pout;
    bool zeroIn;
};
FXD FxSolveBufs fx_solve_bufs(const FxSimDev& S, int phase, int launch) {
    FxSolveBufs r;
    if (phase == 0) {
        const int base = (S.mode == FIREX_PRESSURE_COLD_F32) ? 0 : S.pi;
        r.pin = S.p[(base + launch) & 1];
        r.pout = S.p[(base + launch + 1) & 1];
        r.zeroIn = S.mode == FIREX_PRESSURE_COLD_F32 && launch == 0;
    } else {
        r.pin = S.corr[launch & 1];
        r.pout = S.corr[(launch + 1) & 1];
        r.zeroIn = launch == 0;
    }
    return r;
}

// Finds the simulation owning brick w (start[] ascending, start[nsims] = total).
FXD int fx_find_sim(const int* __restrict__ start, int nsims, int w) {
    int lo = 0, hi = nsims - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(start + mid) <= w) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
