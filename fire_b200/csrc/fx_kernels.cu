// fx_kernels.cu — the Fire-X step passes for sm_100a, batched.
//
// Every step pass takes an FxBatchDev: a device-resident list of simulation descriptors
// (possibly of different grid sizes) and per-shape brick prefix sums. A pass is one
// persistent launch whose CTAs stride over the flat brick list of the whole batch, so a
// single simulation and a batch of uneven ones run the same code, and the launch
// sequence of a step never depends on host-side values (graph-replayable).
//
// Compiled with --fmad=false: each reference expression is the same sequence of IEEE
// operations as in the WGSL source (shaders.ts, pressureShaders.ts).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "fx_internal.h"
#include "fx_jacobi_res.cuh"
#include "fx_sph.cuh"
#include "fx_jacobi_zm.cuh"
#include "fx_jacobi_zm2.cuh"
#include "fx_jacobi_zm2t.cuh"
#include "fx_step_math.cuh"
#include "fx_storage.cuh"

namespace {

// ---- step prologue / epilogue ------------------------------------------------------------
// Time fields of the uniform block for the step about to run (writeUniforms,
// FireXEngine.ts:2049) and the per-step emission jitter (extension): splitmix64 of the
// frame index, 24 random bits, same operations as the host.
__global__ void fxk_step_begin(FxBatchDev* __restrict__ B) {
    // the resident Jacobi's per-box flags start every step at zero (one CTA per simulation)
    for (int s = blockIdx.x; s < B->nsims; s += gridDim.x) {
        FxSimDev* S = B->sims[s];
        for (int i = threadIdx.x; i < 2 * FX_RES_MAX_CTAS; i += blockDim.x) S->sync[FX_RES_FLAGS + i] = 0u;
    }
    if (blockIdx.x != 0) return;
    for (int s = threadIdx.x; s < B->nsims; s += blockDim.x) {
        FxSimDev* S = B->sims[s];
        if (!S->active) continue;
        S->prm.u[U_DT] = (float)S->dt;
        S->prm.u[U_TIME] = (float)S->simTime;
        S->prm.u[6] = (float)S->frame;
        S->prm.u[7] = (float)S->dt;
        uint64_t h = fx_splitmix64(fx_splitmix64(S->seed ^ 0xBB67AE8584CAA73Bull) + (uint64_t)S->frame);
        float u = __fmul_rn((float)(h >> 40), 1.0f / 16777216.0f);
        S->prm.jitter = __fadd_rn(1.0f, __fmul_rn(S->jitterAmp, __fsub_rn(__fmul_rn(2.0f, u), 1.0f)));
    }
}

// Counters after the step (renderOfflineFrameInternal, FireXEngine.ts:681-682) and the
// ping-pong parities of encodeSimulationStep (:2172-2275); copyFlow is a parity flip.
__global__ void fxk_step_end(FxBatchDev* __restrict__ B) {
    for (int s = threadIdx.x; s < B->nsims; s += blockDim.x) {
        FxSimDev* S = B->sims[s];
        if (!S->active) continue;
        S->simTime = S->simTime + S->dt;
        S->frame += 1;
        S->fi ^= 1;
        S->si ^= 1;
        S->pi = (S->mode == FIREX_PRESSURE_COLD_F32) ? (S->P & 1) : (S->pi ^ (S->P & 1));
        if (S->water) S->pti ^= 1;
    }
}

// Per-brick iteration over a batch: calls body(S, brick-in-sim) for every brick of the
// given shape. The owning simulation of consecutive bricks is cached.
template <int SHAPE, class Body>
FXD void fx_for_bricks(const FxBatchDev* __restrict__ B, Body body) {
    const int total = B->total[SHAPE];
    int lo = 0, hi = -1, s = 0;
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
        if (w < lo || w >= hi) {
            s = fx_find_sim(B->start[SHAPE], B->nsims, w);
            lo = __ldg(&B->start[SHAPE][s]);
            hi = __ldg(&B->start[SHAPE][s + 1]);
        }
        const FxSimDev* S = B->sims[s];
        if (!S->active) continue;
        body(*S, w - lo);
    }
}

// ---- simulate (shaders.ts:151-342) -------------------------------------------------------
template <class St>
struct Acc {
    const void* flowIn;
    const void* speciesIn;
    const uint32_t* liq;
    FXD float4 flow(int i) const { return fx_ld_flow(flowIn, i); }
    FXD float4 species(int i) const { return St::ld_species(speciesIn, i); }
    FXD uint32_t liquid(int i) const { return __ldg(liq + i); }
};

// One thread per cell of a 32 x BY x (8 / BY) brick (BY = 2, 4 or 8: the tunable brick
// shape; FX_CELL_BY, 4, by default).
// EARLY: the neighbour terms before the advection (fx_simulate_cell).
template <class St, int BY, bool EARLY>
__global__ void __launch_bounds__(256, 3) fxk_simulate(const FxBatchDev* __restrict__ B) {
    constexpr int BX = FX_CELL_BX, BZ = 256 / (FX_CELL_BX * BY);
    // the simulation's parameter block, the uniform entries of its per-step table and its
    // constant divisors, read by every cell: staged in shared memory when the CTA's brick
    // changes simulation (shared loads instead of about 80 global loads per cell)
    __shared__ FxParams sP;
    __shared__ float sUT[TU_COUNT];
    __shared__ FxDivc sDC[DIVC_COUNT];
    const FxSimDev* cur = nullptr;
    fx_for_bricks<FX_SHAPE_CELL>(B, [&](const FxSimDev& S, int b) {
        if (&S != cur) {      // the same brick, so the same decision, in every thread
            __syncthreads();  // every read of the previous simulation's block is done
            constexpr int nP = sizeof(FxParams) / 4, nD = sizeof(sDC) / 4;
            static_assert(sizeof(FxParams) % 4 == 0 && nP + TU_COUNT + nD <= 1024, "staging words");
            for (int i = threadIdx.x; i < nP + TU_COUNT + nD; i += blockDim.x) {
                if (i < nP) reinterpret_cast<uint32_t*>(&sP)[i] = reinterpret_cast<const uint32_t*>(&S.prm)[i];
                else if (i < nP + TU_COUNT) sUT[i - nP] = S.tab[i - nP];
                else reinterpret_cast<uint32_t*>(sDC)[i - nP - TU_COUNT] = reinterpret_cast<const uint32_t*>(S.divc)[i - nP - TU_COUNT];
            }
            __syncthreads();
            cur = &S;
        }
        const int nbx = (S.X + BX - 1) / BX, nby = (S.Y + BY - 1) / BY;
        const int x = (b % nbx) * BX + threadIdx.x % BX;
        const int y = ((b / nbx) % nby) * BY + (threadIdx.x / BX) % BY;
        const int z = (b / (nbx * nby)) * BZ + threadIdx.x / (BX * BY);
        if (x >= S.X || y >= S.Y || z >= S.Z) return;
        const FxGrid g{S.X, S.Y, S.Z};
        Acc<St> a{S.flow[S.fi], S.species[S.si], S.liquid};
        FxCellOut o = fx_simulate_cell<EARLY>(sP, g, x, y, z, a, S.tab, sUT, sDC);
        const int id = x + S.X * (y + S.Y * z);
        fx_st_flow(S.flow[S.fi ^ 1], id, o.flow);
        St::st_species(S.species[S.si ^ 1], id, o.species);
        S.reaction[id] = o.reaction;
    });
}

// Per-step tables of simulate (fx_table_entry), after fxk_step_begin set the time fields.
__global__ void __launch_bounds__(256) fxk_step_tables(const FxBatchDev* __restrict__ B) {
    fx_for_bricks<FX_SHAPE_TAB>(B, [&](const FxSimDev& S, int b) {
        const int i = b * 256 + (int)threadIdx.x;
        if (i < fx_tab_layout(S.X, S.Y, S.Z).total) S.tab[i] = fx_table_entry(S.prm.u, S.X, S.Y, S.Z, i);
    });
}

// ROW4 brick -> (x0, y, z) of this thread: 4 consecutive cells x0..x0+3. A simulation's
// cells are split into X/4-cell groups in memory order (x fastest; rows are contiguous),
// and brick b holds groups [256 b, 256 b + 256): consecutive threads touch consecutive
// 16-byte segments, and no thread idles except at the end of the simulation.
struct Row4 {
    int x0, y, z;
    bool ok;
};
FXD Row4 fx_row4(const FxSimDev& S, int b) {
    const int gx = S.X >> 2;  // groups < 2^29: 32-bit arithmetic is exact
    const int j = b * FX_ROW4_THREADS + (int)threadIdx.x;
    const int t = j / gx;
    Row4 r;
    r.x0 = (j - t * gx) * 4;
    r.z = t / S.Y;
    r.y = t - r.z * S.Y;
    r.ok = r.z < S.Z;
    return r;
}

// Cells of a ROW4 brick taken lane by lane: the brick's 1024 consecutive cells (memory
// order) are split per warp into 128, and lane l of a warp takes cells l, l+32, l+64,
// l+96 of its 128, so every warp-wide load of a float4 record reads 512 contiguous bytes.
struct Lane4 {
    int c0;       // first cell (memory index) of this lane
    int x, y, z;  // its coordinates
    int n;        // cells of the warp's 128 that exist (the last brick may end early)
};
FXD Lane4 fx_lane4(const FxSimDev& S, int b) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int N = S.X * S.Y * S.Z;  // < 2^31
    const int base = b * (FX_ROW4_THREADS * 4) + w * 128;
    Lane4 r;
    r.c0 = base + lane;
    const int t = r.c0 / S.X;
    r.x = r.c0 - t * S.X;
    r.z = t / S.Y;
    r.y = t - r.z * S.Y;
    r.n = min(128, max(0, N - base));
    return r;
}
// Coordinates of the lane's four cells (32 apart in memory order).
FXD void fx_lane4_coords(const FxSimDev& S, const Lane4& r, int xs[4], int ys[4], int zs[4]) {
    int x = r.x, y = r.y, z = r.z;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        xs[i] = x;
        ys[i] = y;
        zs[i] = z;
        x += 32;
        while (x >= S.X) {
            x -= S.X;
            if (++y == S.Y) {
                y = 0;
                ++z;
            }
        }
    }
}

// ---- computeDivergence (shaders.ts:344-364) ---------------------------------------------
// phase 0: the predicted flow after simulate; phase 1: the primary-projected flow (the
// residual solve's right-hand side). Backward differences with the clamped neighbour
// (the cell itself on the low walls). Every load of the lane's four cells is issued
// before the arithmetic; the x-1 neighbour comes from the next lower lane.
__global__ void __launch_bounds__(256) fxk_divergence(const FxBatchDev* __restrict__ B, int phase) {
    fx_for_bricks<FX_SHAPE_ROW4>(B, [&](const FxSimDev& S, int b) {
        const Lane4 r = fx_lane4(S, b);
        if (r.n <= 0) return;  // warp-uniform
        const int lane = threadIdx.x & 31;
        const float4* __restrict__ flow = reinterpret_cast<const float4*>(phase == 0 ? S.flow[S.fi ^ 1] : S.flow[S.fi]);
        const float3 m = fx_metric(S.prm.u);
        const int X = S.X, XY = S.X * S.Y;
        int xs[4], ys[4], zs[4];
        fx_lane4_coords(S, r, xs, ys, zs);
        float4 cv[4];
        float bottom[4], back[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int c = r.c0 + 32 * i;
            cv[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            bottom[i] = back[i] = 0.0f;
            if (lane + 32 * i < r.n) {
                cv[i] = __ldg(flow + c);
                if (ys[i] > 0) bottom[i] = __ldg(flow + c - X).y;
                if (zs[i] > 0) back[i] = __ldg(flow + c - XY).z;
            }
        }
        // .x of the cell before lane 0's first cell (a previous warp's or brick's cell)
        float prevX = (lane == 0 && xs[0] > 0) ? __ldg(flow + r.c0 - 1).x : 0.0f;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int c = r.c0 + 32 * i;
            const float fromLeft = __shfl_up_sync(0xffffffffu, cv[i].x, 1);
            const float l = xs[i] == 0 ? cv[i].x : (lane > 0 ? fromLeft : prevX);
            prevX = __shfl_sync(0xffffffffu, cv[i].x, 31);
            if (lane + 32 * i < r.n) {
                const float bo = ys[i] > 0 ? bottom[i] : cv[i].y;
                const float ba = zs[i] > 0 ? back[i] : cv[i].z;
                S.div[c] = (cv[i].x - l) * m.x + (cv[i].y - bo) * m.y + (cv[i].z - ba) * m.z;
            }
        }
    });
}

// ---- one Jacobi sweep (solvePressureGlobal, shaders.ts:375-403) --------------------------
// phase 0: primary pressure, sweep index `sweep` of P (warm start from p[pi]; branch C
// starts from zero); phase 1: residual pressure, sweep `sweep` of R, starting from zero.
// A sweep whose input is known to be zero skips its loads: ((wx*(0+0) + ...) - div)/D is
// exactly (0 - div)/D. Storage PT is float or half; the update is FP32.
template <typename PT>
__global__ void __launch_bounds__(256) fxk_jacobi(const FxBatchDev* __restrict__ B, int phase, int launch, int sweep) {
    fx_for_bricks<FX_SHAPE_ROW4>(B, [&](const FxSimDev& S, int b) {
        const int n = phase == 0 ? S.P : S.R;
        if (sweep >= n) return;
        const Row4 r = fx_row4(S, b);
        if (!r.ok) return;
        const FxSolveBufs bufs = fx_solve_bufs(S, phase, launch);
        const void* pin = bufs.pin;
        void* pout = bufs.pout;
        const bool zeroIn = bufs.zeroIn;
        const long long X = S.X, XY = (long long)S.X * S.Y;
        const long long row = (long long)r.y * X + r.z * XY;
        if (r.y == S.Y - 1) {  // the open top is the ambient-pressure boundary
            PStore<PT>::st4(pout, row + r.x0, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
            return;
        }
        const FxJacobiConst c{S.jc[0], S.jc[1], S.jc[2], S.jc[3]};
        const float4 d = __ldg(reinterpret_cast<const float4*>(S.div + row + r.x0));
        float4 o;
        if (zeroIn) {
            o = make_float4((0.0f - d.x) / c.denom, (0.0f - d.y) / c.denom, (0.0f - d.z) / c.denom, (0.0f - d.w) / c.denom);
        } else {
            const long long rowB = (long long)(r.y > 0 ? r.y - 1 : 0) * X + r.z * XY;
            const long long rowT = (long long)(r.y + 1) * X + r.z * XY;
            const long long rowK = (long long)r.y * X + (long long)(r.z > 0 ? r.z - 1 : 0) * XY;
            const long long rowF = (long long)r.y * X + (long long)(r.z < S.Z - 1 ? r.z + 1 : r.z) * XY;
            const float4 pc = PStore<PT>::ld4(pin, row + r.x0);
            const float pl = r.x0 > 0 ? PStore<PT>::ld(pin, row + r.x0 - 1) : pc.x;
            const float pr = r.x0 + 4 < S.X ? PStore<PT>::ld(pin, row + r.x0 + 4) : pc.w;
            const float4 pb = PStore<PT>::ld4(pin, rowB + r.x0);
            const float4 pt = PStore<PT>::ld4(pin, rowT + r.x0);
            const float4 pk = PStore<PT>::ld4(pin, rowK + r.x0);
            const float4 pf = PStore<PT>::ld4(pin, rowF + r.x0);
            o = fx_jacobi4(fx_jacobi_const2(c, S.jcRcp, S.jcFastDiv != 0), pl, pc, pr, pb, pt, pk, pf, d);
        }
        PStore<PT>::st4(pout, row + r.x0, o);
    });
}

// ---- projectVelocity (shaders.ts:461-501, pressureShaders.ts:128-160) ------------------
// phase 0: predicted flow F[1-fi] with the primary pressure -> F[fi];
// phase 1: F[fi] with the residual pressure -> F[1-fi] (the step's result).
// The solve's result sits in the buffer after its last launch; launch counts have the
// parity of the sweep counts (the engine only fuses sweeps when they do), so the result
// buffer is the reference's: p[(base + P) & 1] and corr[R & 1].
// 8 CTAs per SM (32 registers, some spilled): 18 % faster than the 5 that 48 registers allow
// at 508^3 (latency-bound: more loads in flight); the divergence kernel is fastest at 57.
template <typename PT>
__global__ void __launch_bounds__(256, 8) fxk_project(const FxBatchDev* __restrict__ B, int phase) {
    fx_for_bricks<FX_SHAPE_ROW4>(B, [&](const FxSimDev& S, int b) {
        const Lane4 r = fx_lane4(S, b);
        if (r.n <= 0) return;
        const int lane = threadIdx.x & 31;
        const float4* __restrict__ flowIn;
        float4* __restrict__ flowOut;
        const void* p;
        bool zeroP;
        if (phase == 0) {
            flowIn = reinterpret_cast<const float4*>(S.flow[S.fi ^ 1]);
            flowOut = reinterpret_cast<float4*>(S.flow[S.fi]);
            const int base = (S.mode == FIREX_PRESSURE_COLD_F32) ? 0 : S.pi;
            p = S.p[(base + S.P) & 1];
            zeroP = S.mode == FIREX_PRESSURE_COLD_F32 && S.P == 0;
        } else {
            flowIn = reinterpret_cast<const float4*>(S.flow[S.fi]);
            flowOut = reinterpret_cast<float4*>(S.flow[S.fi ^ 1]);
            p = S.corr[S.R & 1];
            zeroP = S.R == 0;
        }
        const float3 m = fx_metric(S.prm.u);
        const int X = S.X, XY = S.X * S.Y;
        int xs[4], ys[4], zs[4];
        fx_lane4_coords(S, r, xs, ys, zs);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (lane + 32 * i < r.n) {
                const int c = r.c0 + 32 * i;
                const int cs = (ys[i] == S.Y - 1) ? c - X : c;  // top row: the projected row below
                const float4 f = __ldg(flowIn + c);
                const float4 src = (cs == c) ? f : __ldg(flowIn + cs);
                float pc = 0.0f, px = 0.0f, pt = 0.0f, pf = 0.0f;
                if (!zeroP) {
                    pc = PStore<PT>::ld(p, cs);
                    px = xs[i] + 1 < X ? PStore<PT>::ld(p, cs + 1) : pc;
                    pt = PStore<PT>::ld(p, cs + X);  // the row above the source row is in the grid
                    pf = zs[i] < S.Z - 1 ? PStore<PT>::ld(p, cs + XY) : pc;
                }
                const float gx = (px - pc) * m.x;
                const float gy = (pt - pc) * m.y;
                const float gz = (pf - pc) * m.z;
                float4 o = make_float4(src.x - gx, src.y - gy, src.z - gz, f.w);
                if (xs[i] == 0 || xs[i] == X - 1) o.x = 0.0f;
                if (zs[i] == 0 || zs[i] == S.Z - 1) o.z = 0.0f;
                if (ys[i] == 0) o.y = 0.0f;
                if (ys[i] == S.Y - 1) o.y = fx_max(0.0f, o.y);
                flowOut[c] = o;
            }
        }
    });
}

// ---- primary projection fused with the residual's divergence -----------------------------
// projectVelocity with the primary pressure (phase 0 above) followed by computeDivergence of
// its result (shaders.ts:344-364; FireXEngine.ts:2256-2257 runs them as two dispatches) in one
// pass: the projected flow is written and its backward divergence stored as the residual
// solve's right-hand side, without reading the projected flow back. The backward neighbours'
// projected components are recomputed with the projection's own operations, so every value
// is bit-identical to the two separate passes:
//   u of the cell before:  the lane before (shuffle), lane 31 of the previous group, or for a
//                          warp's first cell the projection of x - 1 recomputed;
//   v of the row below:    the projection of (x, y - 1, z), never a top-row cell;
//   w of the plane behind: the projection of (x, y, z - 1), from the row below when y is the
//                          top row (the top row copies the projected row below).
// The extra loads (one component of the flow and one pressure value per neighbour) hit
// L1/L2: the rows and planes behind were read by the warps and CTAs before.
#ifndef FX_PROJDIV_MINB
#define FX_PROJDIV_MINB 6  // CTAs per SM the fused projection's registers are budgeted for
#endif
template <typename PT>
struct ProjSrc {
    const float4* __restrict__ flowIn;
    const void* p;
    bool zeroP;
    int X, Y, Z, XY;
    float3 m;
    FXD float pr(int i) const { return zeroP ? 0.0f : PStore<PT>::ld(p, i); }
    // u of cell c = (x, y, z), x in [1, X - 2] (the walls force u = 0 and need no load)
    FXD float u(int c, int x, int y) const {
        if (x == 0 || x == X - 1) return 0.0f;
        const int cs = (y == Y - 1) ? c - X : c;
        const float pc = pr(cs);
        const float px = pr(cs + 1);
        return __ldg(&flowIn[cs].x) - (px - pc) * m.x;
    }
    // v of cell c = (x, y, z) with y <= Y - 2
    FXD float v(int c, int y) const {
        if (y == 0) return 0.0f;
        const float pc = pr(c);
        const float pt = pr(c + X);
        return __ldg(&flowIn[c].y) - (pt - pc) * m.y;
    }
    // w of cell c = (x, y, z) with z <= Z - 2
    FXD float w(int c, int y, int z) const {
        if (z == 0) return 0.0f;
        const int cs = (y == Y - 1) ? c - X : c;
        const float pc = pr(cs);
        const float pf = pr(cs + XY);
        return __ldg(&flowIn[cs].z) - (pf - pc) * m.z;
    }
};

template <typename PT>
__global__ void __launch_bounds__(256, FX_PROJDIV_MINB) fxk_project_div(const FxBatchDev* __restrict__ B) {
    fx_for_bricks<FX_SHAPE_ROW4>(B, [&](const FxSimDev& S, int b) {
        const Lane4 r = fx_lane4(S, b);
        if (r.n <= 0) return;  // warp-uniform
        const int lane = threadIdx.x & 31;
        const int base = (S.mode == FIREX_PRESSURE_COLD_F32) ? 0 : S.pi;
        ProjSrc<PT> src{reinterpret_cast<const float4*>(S.flow[S.fi ^ 1]), S.p[(base + S.P) & 1],
                        S.mode == FIREX_PRESSURE_COLD_F32 && S.P == 0, S.X, S.Y, S.Z, S.X * S.Y, fx_metric(S.prm.u)};
        float4* __restrict__ flowOut = reinterpret_cast<float4*>(S.flow[S.fi]);
        const int X = S.X, XY = S.X * S.Y;
        int xs[4], ys[4], zs[4];
        fx_lane4_coords(S, r, xs, ys, zs);
        // u of the cell before lane 0's first cell (another warp's or brick's cell)
        float prevU = (lane == 0 && xs[0] > 0) ? src.u(r.c0 - 1, xs[0] - 1, ys[0]) : 0.0f;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            // each of the lane's cells is finished in its own iteration: only the u that the
            // next group's first lane needs is carried (registers for more CTAs per SM)
            const bool valid = lane + 32 * i < r.n;
            const int c = r.c0 + 32 * i;
            float4 q = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            float vb = 0.0f, wk = 0.0f;
            if (valid) {
                const int cs = (ys[i] == S.Y - 1) ? c - X : c;  // top row: the projected row below
                const float4 f = __ldg(src.flowIn + c);
                const float4 s = (cs == c) ? f : __ldg(src.flowIn + cs);
                float pc = 0.0f, px = 0.0f, pt = 0.0f, pf = 0.0f;
                if (!src.zeroP) {
                    pc = PStore<PT>::ld(src.p, cs);
                    px = xs[i] + 1 < X ? PStore<PT>::ld(src.p, cs + 1) : pc;
                    pt = PStore<PT>::ld(src.p, cs + X);
                    pf = zs[i] < S.Z - 1 ? PStore<PT>::ld(src.p, cs + XY) : pc;
                }
                const float gx = (px - pc) * src.m.x;
                const float gy = (pt - pc) * src.m.y;
                const float gz = (pf - pc) * src.m.z;
                q = make_float4(s.x - gx, s.y - gy, s.z - gz, f.w);
                if (xs[i] == 0 || xs[i] == X - 1) q.x = 0.0f;
                if (zs[i] == 0 || zs[i] == S.Z - 1) q.z = 0.0f;
                if (ys[i] == 0) q.y = 0.0f;
                if (ys[i] == S.Y - 1) q.y = fx_max(0.0f, q.y);
                flowOut[c] = q;
                vb = ys[i] > 0 ? src.v(c - X, ys[i] - 1) : q.y;
                wk = zs[i] > 0 ? src.w(c - XY, ys[i], zs[i] - 1) : q.z;
            }
            const float fromLeft = __shfl_up_sync(0xffffffffu, q.x, 1);
            const float ul = xs[i] == 0 ? q.x : (lane > 0 ? fromLeft : prevU);
            prevU = __shfl_sync(0xffffffffu, q.x, 31);
            if (valid) S.div[c] = (q.x - ul) * src.m.x + (q.y - vb) * src.m.y + (q.z - wk) * src.m.z;
        }
    });
}

// ---- one Jacobi sweep by z-marching tiles (fx_jacobi_zm.cuh) ---------------------------------
template <typename PT>
__global__ void __launch_bounds__(FX_ZM_THREADS, 3) fxk_jacobi_zm(const FxBatchDev* __restrict__ B, int phase, int launch,
                                                               int sweep, int zc) {
    extern __shared__ __align__(16) unsigned char fx_zm_dyn[];
    FxZmSmem<PT>& sm = *reinterpret_cast<FxZmSmem<PT>*>(fx_zm_dyn);
    fx_for_bricks<FX_SHAPE_ZM>(B, [&](const FxSimDev& S, int b) {
        const int n = phase == 0 ? S.P : S.R;
        if (sweep >= n) return;
        const int TX = fx_zm_tile_w(S.X), TY = FX_ZM_CELLS / TX;
        const int ntx = (S.X + TX - 1) / TX, nty = (S.Y + TY - 1) / TY;
        const int tx = b % ntx, ty = (b / ntx) % nty, zci = b / (ntx * nty);
        const int z0 = zci * zc, z1 = min(S.Z, z0 + zc);
        const FxSolveBufs bufs = fx_solve_bufs(S, phase, launch);
        const PT* pin = reinterpret_cast<const PT*>(bufs.pin);
        PT* pout = reinterpret_cast<PT*>(bufs.pout);
        const int x0 = tx * TX, y0 = ty * TY;
        if (bufs.zeroIn) {
            if (TX == 128) fx_zm_tile<PT, true, 128>(&S, pin, pout, x0, y0, z0, z1, sm);
            else if (TX == 64) fx_zm_tile<PT, true, 64>(&S, pin, pout, x0, y0, z0, z1, sm);
            else fx_zm_tile<PT, true, 32>(&S, pin, pout, x0, y0, z0, z1, sm);
        } else {
            if (TX == 128) fx_zm_tile<PT, false, 128>(&S, pin, pout, x0, y0, z0, z1, sm);
            else if (TX == 64) fx_zm_tile<PT, false, 64>(&S, pin, pout, x0, y0, z0, z1, sm);
            else fx_zm_tile<PT, false, 32>(&S, pin, pout, x0, y0, z0, z1, sm);
        }
    });
}

// ---- two Jacobi sweeps per pass by z-marching tiles (fx_jacobi_zm2.cuh) ------------------------
template <typename PT, bool ROUND>
__global__ void __launch_bounds__(FX_Z2_THREADS, FX_Z2_MINB) fxk_jacobi_zm2(const FxBatchDev* __restrict__ B, int phase, int launch,
                                                                int zc) {
    extern __shared__ __align__(16) unsigned char fx_z2_dyn[];
    FxZ2Smem<PT>& sm = *reinterpret_cast<FxZ2Smem<PT>*>(fx_z2_dyn);
    fx_for_bricks<FX_SHAPE_COL>(B, [&](const FxSimDev& S, int b) {
        const int ntx = (S.X + FX_Z2_TX - 1) / FX_Z2_TX, nty = (S.Y + FX_Z2_TY - 1) / FX_Z2_TY;
        const int tx = b % ntx, ty = (b / ntx) % nty, zci = b / (ntx * nty);
        const int z0 = zci * zc, z1 = min(S.Z, z0 + zc);
        const FxSolveBufs bufs = fx_solve_bufs(S, phase, launch);
        const PT* pin = reinterpret_cast<const PT*>(bufs.pin);
        PT* pout = reinterpret_cast<PT*>(bufs.pout);
        if (bufs.zeroIn) fx_zm2_tile<PT, true, ROUND>(S, pin, pout, tx * FX_Z2_TX, ty * FX_Z2_TY, z0, z1, sm);
        else fx_zm2_tile<PT, false, ROUND>(S, pin, pout, tx * FX_Z2_TX, ty * FX_Z2_TY, z0, z1, sm);
    });
}

// ---- two Jacobi sweeps per pass, planes staged by TMA (fx_jacobi_zm2t.cuh), FP32 pressure --------
__global__ void __launch_bounds__(FX_Z2_THREADS, FX_Z2_MINB) fxk_jacobi_zm2t(const FxBatchDev* __restrict__ B, int phase,
                                                                int launch, int zc) {
    extern __shared__ __align__(128) unsigned char fx_t2_dyn[];
    // the slots must start on 128-byte boundaries: align the dynamic window (128 bytes spare)
    FxT2Smem& sm = *reinterpret_cast<FxT2Smem*>((reinterpret_cast<uintptr_t>(fx_t2_dyn) + 127) & ~(uintptr_t)127);
    if (threadIdx.x == 0) {
        for (int i = 0; i < FX_T2_SLOTS; ++i) fx_mbar_init(&sm.bar[i], 1);
        sm.err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    unsigned phases = 0;  // parity of each slot's next barrier phase (the same in every thread)
    const int total = B->total[FX_SHAPE_COL];
    int lo = 0, hi = -1, si = 0;
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
        if (w < lo || w >= hi) {
            si = fx_find_sim(B->start[FX_SHAPE_COL], B->nsims, w);
            lo = __ldg(&B->start[FX_SHAPE_COL][si]);
            hi = __ldg(&B->start[FX_SHAPE_COL][si + 1]);
        }
        const FxSimDev& S = *B->sims[si];
        if (!S.active) continue;
        const int b = w - lo;
        const int ntx = (S.X + FX_Z2_TX - 1) / FX_Z2_TX, nty = (S.Y + FX_Z2_TY - 1) / FX_Z2_TY;
        const int tx = b % ntx, ty = (b / ntx) % nty, zci = b / (ntx * nty);
        const int z0 = zci * zc, z1 = min(S.Z, z0 + zc);
        const FxSolveBufs bufs = fx_solve_bufs(S, phase, launch);
        float* pout = reinterpret_cast<float*>(bufs.pout);
        const bool ok = bufs.zeroIn
                            ? fx_zm2t_tile<true>(S, nullptr, pout, tx * FX_Z2_TX, ty * FX_Z2_TY, z0, z1, sm, phases)
                            : fx_zm2t_tile<false>(S, fx_t2_map_of(S, bufs.pin), pout, tx * FX_Z2_TX, ty * FX_Z2_TY, z0,
                                                  z1, sm, phases);
        if (!ok) {  // a barrier wait ran out: report it and stop this CTA
            if (threadIdx.x == 0) atomicExch(S.sync + 2, 1u);
            return;
        }
    }
}

// Counts the floats x for which fx_div_by_const(x, d, rcp) differs from the IEEE
// quotient x / d (every bit pattern, 2^32 of them; any NaN matches any NaN).
__global__ void fxk_check_div(float d, float rcp, float lo, float hi, unsigned long long* __restrict__ mismatches) {
    unsigned long long bad = 0;
    const unsigned long long n = 1ull << 32;
    for (unsigned long long b = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; b < n;
         b += (unsigned long long)gridDim.x * blockDim.x) {
        const float x = __uint_as_float((unsigned)b);
        const float a = fx_div_range(x, d, rcp, lo, hi), e = __fdiv_rn(x, d);
        bad += (__float_as_uint(a) != __float_as_uint(e)) && !(a != a && e != e);  // NaN == NaN
    }
    if (bad) atomicAdd(mismatches, bad);
}

// ---- single-simulation utilities -----------------------------------------------------------
// initializeFields (shaders.ts:135-149) plus the seeded velocity noise extension; writes
// flow[fi] and species[si] of the descriptor.
template <class St>
__global__ void fxk_init(const FxSimDev* __restrict__ S, float tAmbient, float oxygen, float noise) {
    const long long n = (long long)S->X * S->Y * S->Z;
    void* flow = S->flow[S->fi];
    void* species = S->species[S->si];
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < n; id += (long long)gridDim.x * blockDim.x) {
        float4 f = make_float4(0.0f, 0.0f, 0.0f, tAmbient);
        if (noise > 0.0f) {
            f.x = fx_velocity_noise(S->seed, (uint64_t)id, 0, noise);
            f.y = fx_velocity_noise(S->seed, (uint64_t)id, 1, noise);
            f.z = fx_velocity_noise(S->seed, (uint64_t)id, 2, noise);
        }
        fx_st_flow(flow, id, f);
        St::st_species(species, id, make_float4(0.0f, fx_max(oxygen, 0.0f), 0.0f, 0.0f));
    }
}

__global__ void fxk_emitter_mask(const FxSimDev* __restrict__ S, uint8_t* __restrict__ mask) {
    const long long n = (long long)S->X * S->Y * S->Z;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < n; id += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(id % S->X);
        const int y = (int)((id / S->X) % S->Y);
        const int z = (int)(id / ((long long)S->X * S->Y));
        uint8_t m = 0;
        if (S->prm.emitter_mode == FIREX_EMITTER_SPHERES)
            for (int s = 0; s < S->prm.num_spheres; ++s)
                if (fx_sphere_inside(S->prm.spheres[s], x, y, z)) m = 1;
        mask[id] = m;
    }
}

// ---- SPH droplets and liquid deposition (fx_sph.cuh), before simulate --------------------
// Members whose water runs: clear the liquid field, then density, integration (droplets
// part[pti] -> part[pti ^ 1]) and deposition; step_end flips pti.
// ---- droplets (FIREX_PARTICLE_WGSL, shaders.ts:514-825) -----------------------------------
// Two launches per step: the liquid clear of every spraying member with the droplet
// densities, then integration with each droplet's deposit (a droplet deposits only its own
// old and new state, so it needs no other droplet's result).
__global__ void __launch_bounds__(FX_SPH_THREADS) fxk_sph_density(const FxBatchDev* __restrict__ B) {
    fx_for_bricks<FX_SHAPE_ROW4>(B, [&](const FxSimDev& S, int b) {  // encoder.clearBuffer(liquid)
        if (!S.water) return;
        static_assert(FX_SPH_THREADS == FX_ROW4_THREADS, "one ROW4 brick per block");
        const long long i = (long long)b * (FX_ROW4_THREADS * 4) + 4 * threadIdx.x;
        const long long n = (long long)S.X * S.Y * S.Z;
        if (i < n) *reinterpret_cast<uint4*>(S.liquid + i) = make_uint4(0u, 0u, 0u, 0u);  // n % 4 == 0
    });
    fx_for_bricks<FX_SHAPE_PART>(B, [&](const FxSimDev& S, int b) {
        const int i = b * FX_SPH_DROPLETS + (threadIdx.x >> 5), lane = threadIdx.x & 31;
        if (i >= S.np) return;  // warp-uniform
        const fxsph::Ctx c{S.prm.u, S.X, S.Y, S.Z};
        const float4 d = fxsph::density_warp(c, S.np, S.part[S.pti], i, lane);
        if (lane == 0) S.pdens[i] = d;
    });
}
__global__ void __launch_bounds__(FX_SPH_THREADS) fxk_sph_integrate(const FxBatchDev* __restrict__ B) {
    fx_for_bricks<FX_SHAPE_PART>(B, [&](const FxSimDev& S, int b) {
        const int i = b * FX_SPH_DROPLETS + (threadIdx.x >> 5), lane = threadIdx.x & 31;
        if (i >= S.np) return;  // warp-uniform
        const fxsph::Ctx c{S.prm.u, S.X, S.Y, S.Z};
        const float4* pin = S.part[S.pti];
        float4 oa, om;
        fxsph::integrate_warp(c, S.np, pin, S.pdens, reinterpret_cast<const float4*>(S.flow[S.fi]), i, lane, oa, om);
        if (lane == 0) {
            S.part[S.pti ^ 1][2 * i] = oa;
            S.part[S.pti ^ 1][2 * i + 1] = om;
        }
        fxsph::deposit_warp(c, __ldg(pin + 2 * i), __ldg(pin + 2 * i + 1), oa, om, S.liquid, lane);
    });
}

// ---- render-field packing (storePackedFields, qualityShaders.ts:37-75) --------------------
// The three rgba16float volumes of the canonical state as FP16 (round to nearest even):
// flow (u, v, w, clamp((T - 300) / 2600, 0, 1)), chemistry (max(species, 0)) and media
// (reaction, soot, liquid, display value). In view 7 the display value is the divergence of
// the canonical flow the presentation computes (FireXEngine.ts:2588-2596), 0 on the outer
// shell. Headless device buffers stand in for the reference's textures.
FXD uint2 fx_half4(float a, float b, float c, float d) {
    const __half2 lo = __floats2half2_rn(a, b), hi = __floats2half2_rn(c, d);
    uint2 r;
    r.x = *reinterpret_cast<const uint32_t*>(&lo);
    r.y = *reinterpret_cast<const uint32_t*>(&hi);
    return r;
}
FXD void fx_pack_cell(const FxSimDev& S, int id, int x, int y, int z, bool view7, const float3& m) {
    const float4* flow = reinterpret_cast<const float4*>(S.flow[S.fi]);
    const float4 f = __ldg(flow + id);
    const float4 sr = S.storage == FX_STORAGE_MIXED ? StMixed::ld_species(S.species[S.si], id)
                                                    : StF32::ld_species(S.species[S.si], id);
    const float4 sp = make_float4(fx_max(sr.x, 0.0f), fx_max(sr.y, 0.0f), fx_max(sr.z, 0.0f), fx_max(sr.w, 0.0f));
    const float reaction = fx_clamp(__ldg(S.reaction + id), 0.0f, 4.0f);
    const float richness = fx_clamp(sp.x / fx_max(sp.x + sp.y * 0.25f, FC(0.0001)), 0.0f, 1.0f);
    const float soot = sp.z * fx_smoothstep(0.25f, FC(0.82), richness);
    const float liq = (float)__ldg(S.liquid + id) * FC(3.4 / 4096.0);
    float disp = fx_max(fx_max(reaction, soot), fx_max(liq, fx_max(sp.w, fx_smoothstep(420.0f, 700.0f, f.w))));
    if (view7) {
        const bool shell = x == 0 || y == 0 || z == 0 || x + 1 >= S.X || y + 1 >= S.Y || z + 1 >= S.Z;
        if (shell) {
            disp = 0.0f;
        } else {
            const float l = __ldg(flow + id - 1).x;
            const float bo = __ldg(flow + id - S.X).y;
            const float ba = __ldg(flow + id - S.X * S.Y).z;
            disp = (f.x - l) * m.x + (f.y - bo) * m.y + (f.z - ba) * m.z;
        }
    }
    S.render[0][id] = fx_half4(f.x, f.y, f.z, fx_clamp((f.w - 300.0f) / 2600.0f, 0.0f, 1.0f));
    S.render[1][id] = fx_half4(sp.x, sp.y, sp.z, sp.w);
    S.render[2][id] = fx_half4(reaction, soot, liq, disp);
}
FXD bool fx_view7(const float* u) { return (unsigned)fx_clamp(rintf(u[U_VIEW_MODE]), 0.0f, 7.0f) == 7u; }

// One simulation's volumes (a read of a render field).
__global__ void fxk_pack_sim(const FxSimDev* __restrict__ Sp) {
    const FxSimDev& S = *Sp;
    const int n = S.X * S.Y * S.Z;
    const float3 m = fx_metric(S.prm.u);
    const bool v7 = fx_view7(S.prm.u);
    for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < n; id += gridDim.x * blockDim.x) {
        const int x = id % S.X, t = id / S.X, y = t % S.Y, z = t / S.Y;
        fx_pack_cell(S, id, x, y, z, v7, m);
    }
}

// Every member that packs each step, after the step's end (canonical buffers current).
__global__ void __launch_bounds__(256) fxk_pack_batch(const FxBatchDev* __restrict__ B) {
    fx_for_bricks<FX_SHAPE_ROW4>(B, [&](const FxSimDev& S, int b) {
        if (!S.renderPack) return;
        const Lane4 r = fx_lane4(S, b);
        if (r.n <= 0) return;
        const int lane = threadIdx.x & 31;
        const float3 m = fx_metric(S.prm.u);
        const bool v7 = fx_view7(S.prm.u);
        int xs[4], ys[4], zs[4];
        fx_lane4_coords(S, r, xs, ys, zs);
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (lane + 32 * i < r.n) fx_pack_cell(S, r.c0 + 32 * i, xs[i], ys[i], zs[i], v7, m);
    });
}

// Divergence of the canonical flow F[fi] into out (the FINAL_DIVERGENCE field).
__global__ void fxk_final_divergence(const FxSimDev* __restrict__ S, float* __restrict__ out) {
    const long long n = (long long)S->X * S->Y * S->Z;
    const float3 m = fx_metric(S->prm.u);
    const void* flow = S->flow[S->fi];
    const FxGrid g{S->X, S->Y, S->Z};
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < n; id += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(id % S->X);
        const int y = (int)((id / S->X) % S->Y);
        const int z = (int)(id / ((long long)S->X * S->Y));
        const float4 c = fx_ld_flow(flow, id);
        const float l = fx_ld_flow(flow, g.idx(x - 1, y, z)).x;
        const float bo = fx_ld_flow(flow, g.idx(x, y - 1, z)).y;
        const float ba = fx_ld_flow(flow, g.idx(x, y, z - 1)).z;
        out[id] = (c.x - l) * m.x + (c.y - bo) * m.y + (c.z - ba) * m.z;
    }
}

// Post-projection divergence norm over interior cells (the one-cell shell excluded,
// qualityShaders.ts:47-57): per-block FP64 partial (sum of squares, max abs), then a
// fixed-order final reduction (deterministic).
__global__ void __launch_bounds__(256) fxk_norm_partial(const FxSimDev* __restrict__ S, double* __restrict__ partial) {
    const float3 m = fx_metric(S->prm.u);
    const void* flow = S->flow[S->fi];
    const long long X = S->X, XY = (long long)S->X * S->Y;
    const long long nInt = (long long)(S->X - 2) * (S->Y - 2) * (S->Z - 2);
    double ss = 0.0, mx = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nInt; k += (long long)gridDim.x * blockDim.x) {
        const int x = 1 + (int)(k % (S->X - 2));
        const int y = 1 + (int)((k / (S->X - 2)) % (S->Y - 2));
        const int z = 1 + (int)(k / ((long long)(S->X - 2) * (S->Y - 2)));
        const long long id = x + X * y + XY * z;
        const float4 c = fx_ld_flow(flow, id);
        const float d = (c.x - fx_ld_flow(flow, id - 1).x) * m.x + (c.y - fx_ld_flow(flow, id - X).y) * m.y +
                        (c.z - fx_ld_flow(flow, id - XY).z) * m.z;
        const double dd = (double)d;
        ss += dd * dd;
        mx = fmax(mx, fabs(dd));
    }
    __shared__ double s_ss[256], s_mx[256];
    const int t = threadIdx.x;
    s_ss[t] = ss;
    s_mx[t] = mx;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (t < w) {
            s_ss[t] += s_ss[t + w];
            s_mx[t] = fmax(s_mx[t], s_mx[t + w]);
        }
        __syncthreads();
    }
    if (t == 0) {
        partial[2 * blockIdx.x] = s_ss[0];
        partial[2 * blockIdx.x + 1] = s_mx[0];
    }
}

// ---- every sweep of a Jacobi phase in one cooperative launch (fx_jacobi_res.cuh) --------
// VARIANT: 0 column, 1 faces-first, 2 faces-first for small boxes, 3 faces-first with
// interior columns, 4 variant 3 with a copy warp (FP32 pressure) (fx_jacobi_res.cuh).
// EPI (variant 4, residual phase): the projection epilogue (fx_res_project_epi).
template <typename PT, int VARIANT, bool EPI = false>
__global__ void __launch_bounds__(FX_RES_THREADS, 1) fxk_jacobi_res(const FxBatchDev* __restrict__ B, int phase) {
    extern __shared__ float4 fx_res_smem[];
    const int w = blockIdx.x;
    if (w >= B->total[FX_SHAPE_RES]) return;
    const int si = fx_find_sim(B->start[FX_SHAPE_RES], B->nsims, w);
    const FxSimDev& S = *B->sims[si];
    if (!S.active) return;
    float* sm = reinterpret_cast<float*>(fx_res_smem);
    const int b = w - B->start[FX_SHAPE_RES][si];
    if (VARIANT == 1) fx_res_box_early<PT, sizeof(PT) == 2, FX_RES_MAXI>(S, B->res[si], b, phase, sm);
    else if (VARIANT == 2) fx_res_box_early<PT, sizeof(PT) == 2, FX_RES_MAXI_SMALL>(S, B->res[si], b, phase, sm);
    else if (VARIANT == 3) fx_res_box_v3<PT, sizeof(PT) == 2, false>(S, B->res[si], b, phase, sm);
    else if (VARIANT == 4) {
        if constexpr (sizeof(PT) == 4) fx_res_box_v3<float, false, true, EPI>(S, B->res[si], b, phase, sm);
    }
    else fx_res_box_col<PT, sizeof(PT) == 2>(S, B->res[si], b, phase, sm);
}

__global__ void fxk_norm_final(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
    __shared__ double s_ss[256], s_mx[256];
    const int t = threadIdx.x;
    double ss = 0.0, mx = 0.0;
    for (int b = t; b < nblocks; b += blockDim.x) {
        ss += partial[2 * b];
        mx = fmax(mx, partial[2 * b + 1]);
    }
    s_ss[t] = ss;
    s_mx[t] = mx;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (t < w) {
            s_ss[t] += s_ss[t + w];
            s_mx[t] = fmax(s_mx[t], s_mx[t + w]);
        }
        __syncthreads();
    }
    if (t == 0) {
        out[0] = sqrt(s_ss[0]);
        out[1] = s_mx[0];
    }
}

}  // namespace

// ---- launch wrappers ---------------------------------------------------------------------------
static int g_num_sms = 0;
static int num_sms() {
    if (!g_num_sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    return g_num_sms;
}

// Grid sizing. Stencil passes launch one CTA per brick (the hardware keeps every SM
// full and overlaps CTAs' memory latency); FX_PERSISTENT_ROW4 switches them to a
// persistent grid of full residency that strides over the bricks.
static int g_row4_persistent = -1;
static bool row4_persistent() {
    if (g_row4_persistent < 0) {
        const char* e = getenv("FX_PERSISTENT_ROW4");
        g_row4_persistent = (e && e[0] == '1') ? 1 : 0;
    }
    return g_row4_persistent == 1;
}
static int row4_grid(int g, int bricks) { return row4_persistent() ? (bricks < g ? bricks : g) : bricks; }

// Persistent grid: enough CTAs for full residency, never more than the brick count.
static int persistent_grid(const void* kernel, int threads, int bricks) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0);
    if (per_sm <= 0) per_sm = 1;
    long long g = (long long)per_sm * num_sms();
    if (bricks > 0 && bricks < g) g = bricks;
    return (int)(g < 1 ? 1 : g);
}

void fx_launch_step_begin(cudaStream_t s, FxBatchDev* B) { fxk_step_begin<<<32, 256, 0, s>>>(B); }
void fx_launch_step_end(cudaStream_t s, FxBatchDev* B) { fxk_step_end<<<1, 256, 0, s>>>(B); }
void fx_launch_step_tables(cudaStream_t s, const FxBatchDev* B, int bricks) {
    fxk_step_tables<<<bricks > 0 ? bricks : 1, 256, 0, s>>>(B);
}

template <class St, int BY, bool EARLY>
static void launch_simulate(cudaStream_t s, const FxBatchDev* B, int bricks) {
    static int g = persistent_grid((const void*)fxk_simulate<St, BY, EARLY>, 256, 1 << 30);
    fxk_simulate<St, BY, EARLY><<<bricks < g ? bricks : g, 256, 0, s>>>(B);
}

template <class St, bool EARLY>
static void launch_simulate_shape(cudaStream_t s, int by, const FxBatchDev* B, int bricks) {
    if (by == 2) launch_simulate<St, 2, EARLY>(s, B, bricks);
    else if (by == 8) launch_simulate<St, 8, EARLY>(s, B, bricks);
    else launch_simulate<St, 4, EARLY>(s, B, bricks);
}

void fx_launch_simulate(cudaStream_t s, int storage, int by, bool early, const FxBatchDev* B, int bricks) {
    if (storage == FX_STORAGE_MIXED) {  // the reference order only (measured faster for mixed storage)
        launch_simulate_shape<StMixed, false>(s, by, B, bricks);
    } else {
        if (early) launch_simulate_shape<StF32, true>(s, by, B, bricks);
        else launch_simulate_shape<StF32, false>(s, by, B, bricks);
    }
}

void fx_launch_divergence(cudaStream_t s, const FxBatchDev* B, int bricks, int phase) {
    static int g = persistent_grid((const void*)fxk_divergence, 256, 1 << 30);
    fxk_divergence<<<row4_grid(g, bricks), 256, 0, s>>>(B, phase);
}

void fx_launch_jacobi(cudaStream_t s, bool half, const FxBatchDev* B, int bricks, int phase, int launch, int sweep) {
    if (half) {
        static int g = persistent_grid((const void*)fxk_jacobi<__half>, 256, 1 << 30);
        fxk_jacobi<__half><<<row4_grid(g, bricks), 256, 0, s>>>(B, phase, launch, sweep);
    } else {
        static int g = persistent_grid((const void*)fxk_jacobi<float>, 256, 1 << 30);
        fxk_jacobi<float><<<row4_grid(g, bricks), 256, 0, s>>>(B, phase, launch, sweep);
    }
}

template <typename PT>
static void launch_zm(cudaStream_t s, const FxBatchDev* B, int bricks, int phase, int launch, int sweep, int zc) {
    static const int g = [] {
        cudaFuncSetAttribute((const void*)fxk_jacobi_zm<PT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(FxZmSmem<PT>));
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fxk_jacobi_zm<PT>, FX_ZM_THREADS,
                                                      sizeof(FxZmSmem<PT>));
        return (per_sm > 0 ? per_sm : 1) * num_sms();
    }();
    fxk_jacobi_zm<PT><<<row4_grid(g, bricks), FX_ZM_THREADS, sizeof(FxZmSmem<PT>), s>>>(B, phase, launch, sweep, zc);
}

void fx_launch_jacobi_zm(cudaStream_t s, bool half, const FxBatchDev* B, int bricks, int phase, int launch, int sweep,
                         int zc) {
    if (half) launch_zm<__half>(s, B, bricks, phase, launch, sweep, zc);
    else launch_zm<float>(s, B, bricks, phase, launch, sweep, zc);
}

template <typename PT, bool ROUND>
static void launch_zm2(cudaStream_t s, const FxBatchDev* B, int bricks, int phase, int launch, int zc) {
    static int g = [] {
        cudaFuncSetAttribute((const void*)fxk_jacobi_zm2<PT, ROUND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(FxZ2Smem<PT>));
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fxk_jacobi_zm2<PT, ROUND>, FX_Z2_THREADS,
                                                      sizeof(FxZ2Smem<PT>));
        return (per_sm > 0 ? per_sm : 1) * num_sms();
    }();
    fxk_jacobi_zm2<PT, ROUND><<<bricks < g ? bricks : g, FX_Z2_THREADS, sizeof(FxZ2Smem<PT>), s>>>(B, phase, launch, zc);
}

#ifndef FX_T2_L2_PROMOTION
#define FX_T2_L2_PROMOTION CU_TENSOR_MAP_L2_PROMOTION_L2_128B
#endif
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link-time dependency on
// the driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        cudaGetLastError();
    });
    return fn;
}

// A 3-D FP32 map of an X x Y x Z field (x fastest) with boxes of FX_Z2_COLS x boxY x 1 cells:
// row stride X * 4 bytes (a multiple of 16: X is a multiple of 4), out-of-bound cells read 0.
static bool map_field(EncodeTiledFn fn, CUtensorMap* m, void* base, int X, int Y, int Z, int boxY) {
    const cuuint64_t dims[3] = {(cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)Z};
    const cuuint64_t strides[2] = {(cuuint64_t)X * 4, (cuuint64_t)X * (cuuint64_t)Y * 4};
    const cuuint32_t box[3] = {FX_Z2_COLS, (cuuint32_t)boxY, 1};
    const cuuint32_t elem[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, FX_T2_L2_PROMOTION, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool fx_make_tensor_maps(FxSimDev* h) {
    h->tmapOk = 0;
    EncodeTiledFn fn = encode_tiled();
    if (!fn || h->mode == FIREX_PRESSURE_F16 || (h->X & 3) != 0) return false;
    void* bufs[4] = {h->p[0], h->p[1], h->corr[0], h->corr[1]};
    for (int i = 0; i < 4; ++i)
        if (!map_field(fn, &h->tmap[FX_TM_P0 + i], bufs[i], h->X, h->Y, h->Z, FX_T2_PBOX_Y)) return false;
    if (!map_field(fn, &h->tmap[FX_TM_DIV], h->div, h->X, h->Y, h->Z, FX_T2_DBOX_Y)) return false;
    h->tmapOk = 1;
    return true;
}

static void launch_zm2t(cudaStream_t s, const FxBatchDev* B, int bricks, int phase, int launch, int zc) {
    constexpr int smem = (int)sizeof(FxT2Smem) + 128;
    static int g = [] {
        cudaFuncSetAttribute((const void*)fxk_jacobi_zm2t, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fxk_jacobi_zm2t, FX_Z2_THREADS, smem);
        return (per_sm > 0 ? per_sm : 1) * num_sms();
    }();
    fxk_jacobi_zm2t<<<bricks < g ? bricks : g, FX_Z2_THREADS, smem, s>>>(B, phase, launch, zc);
}

bool fx_launch_jacobi_tb(cudaStream_t s, int pmode, int k, const FxBatchDev* B, int bricks, int phase, int launch, int zc,
                         bool tma) {
    switch (k) {
        case 2:  // two sweeps per pass: the z-marching form
            if (pmode == FX_TB_F32 && tma) launch_zm2t(s, B, bricks, phase, launch, zc);
            else if (pmode == FX_TB_F32) launch_zm2<float, false>(s, B, bricks, phase, launch, zc);
            else if (pmode == FX_TB_F16_ROUND) launch_zm2<__half, true>(s, B, bricks, phase, launch, zc);
            else launch_zm2<__half, false>(s, B, bricks, phase, launch, zc);
            return true;
    }
    return false;
}

template <typename PT, int VARIANT>
static const void* res_fn() {
    return (const void*)fxk_jacobi_res<PT, VARIANT>;
}
static const void* res_kernel(bool half, int variant) {
    switch (variant) {
        case 4: return half ? nullptr : res_fn<float, 4>();
        case 1: return half ? res_fn<__half, 1>() : res_fn<float, 1>();
        case 2: return half ? res_fn<__half, 2>() : res_fn<float, 2>();
        case 3: return half ? res_fn<__half, 3>() : res_fn<float, 3>();
        default: return half ? res_fn<__half, 0>() : res_fn<float, 0>();
    }
}

// Most CTAs of resident-Jacobi variant `variant` that one cooperative launch can keep
// resident (0: the variant cannot run, e.g. variant 4 with FP16 pressure).
int fx_res_capacity(bool half, int variant) {
    const void* fn = res_kernel(half, variant);
    if (!fn) return 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, FX_RES_SMEM_MAX) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, FX_RES_THREADS, FX_RES_SMEM_MAX) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return per_sm * num_sms();
}

cudaError_t fx_launch_jacobi_res(cudaStream_t s, bool half, int variant, const FxBatchDev* B, int ctas, int phase,
                                 int smem, bool epi) {
    const void* fn = (epi && variant == 4 && !half) ? (const void*)fxk_jacobi_res<float, 4, true> : res_kernel(half, variant);
    if (!fn) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, FX_RES_SMEM_MAX);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3(FX_RES_THREADS);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* args[] = {(void*)&B, (void*)&phase};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

void fx_launch_project(cudaStream_t s, bool half, const FxBatchDev* B, int bricks, int phase) {
    if (half) {
        static int g = persistent_grid((const void*)fxk_project<__half>, 256, 1 << 30);
        fxk_project<__half><<<row4_grid(g, bricks), 256, 0, s>>>(B, phase);
    } else {
        static int g = persistent_grid((const void*)fxk_project<float>, 256, 1 << 30);
        fxk_project<float><<<row4_grid(g, bricks), 256, 0, s>>>(B, phase);
    }
}

void fx_launch_project_div(cudaStream_t s, bool half, const FxBatchDev* B, int bricks) {
    if (half) {
        static int g = persistent_grid((const void*)fxk_project_div<__half>, 256, 1 << 30);
        fxk_project_div<__half><<<row4_grid(g, bricks), 256, 0, s>>>(B);
    } else {
        static int g = persistent_grid((const void*)fxk_project_div<float>, 256, 1 << 30);
        fxk_project_div<float><<<row4_grid(g, bricks), 256, 0, s>>>(B);
    }
}

void fx_launch_init(cudaStream_t s, int storage, const FxSimDev* S, float tAmbient, float oxygen, float noise) {
    if (storage == FX_STORAGE_MIXED) fxk_init<StMixed><<<num_sms() * 8, 256, 0, s>>>(S, tAmbient, oxygen, noise);
    else fxk_init<StF32><<<num_sms() * 8, 256, 0, s>>>(S, tAmbient, oxygen, noise);
}

void fx_launch_emitter_mask(cudaStream_t s, const FxSimDev* S, uint8_t* mask) {
    fxk_emitter_mask<<<num_sms() * 8, 256, 0, s>>>(S, mask);
}

void fx_launch_sph(cudaStream_t s, const FxBatchDev* B, int rowBricks, int partBricks) {
    static int g = persistent_grid((const void*)fxk_sph_density, FX_SPH_THREADS, 1 << 30);
    fxk_sph_density<<<std::max(partBricks, row4_grid(g, rowBricks)), FX_SPH_THREADS, 0, s>>>(B);
    fxk_sph_integrate<<<partBricks, FX_SPH_THREADS, 0, s>>>(B);
}

void fx_launch_pack_sim(cudaStream_t s, const FxSimDev* S) { fxk_pack_sim<<<num_sms() * 8, 256, 0, s>>>(S); }
void fx_launch_pack_batch(cudaStream_t s, const FxBatchDev* B, int bricks) {
    static int g = persistent_grid((const void*)fxk_pack_batch, 256, 1 << 30);
    fxk_pack_batch<<<row4_grid(g, bricks), 256, 0, s>>>(B);
}

void fx_launch_final_divergence(cudaStream_t s, const FxSimDev* S, float* out) {
    fxk_final_divergence<<<num_sms() * 8, 256, 0, s>>>(S, out);
}

int fx_norm_partial_blocks(long long cells) {
    long long b = (cells + 255) / 256;
    const long long cap = 148LL * 8;
    return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

void fx_launch_divergence_norm(cudaStream_t s, const FxSimDev* S, long long cells, double* partial, double* out) {
    const int nb = fx_norm_partial_blocks(cells);
    fxk_norm_partial<<<nb, 256, 0, s>>>(S, partial);
    fxk_norm_final<<<1, 256, 0, s>>>(partial, nb, out);
}

// Descriptor uploads travel as kernel arguments: no host staging buffer has to outlive
// the call, and the copy is ordered on the stream like any other pass.
namespace {
__global__ void fxk_upload_desc(FxSimDev v, FxSimDev* __restrict__ dst) {
    const int* src = reinterpret_cast<const int*>(&v);
    int* d = reinterpret_cast<int*>(dst);
    for (int i = threadIdx.x; i < (int)(sizeof(FxSimDev) / 4); i += blockDim.x) d[i] = src[i];
}
}  // namespace

void fx_launch_upload_desc(cudaStream_t s, const FxSimDev& host, FxSimDev* dev) { fxk_upload_desc<<<1, 128, 0, s>>>(host, dev); }

void fx_launch_upload_batch(cudaStream_t s, const FxBatchDev& host, FxBatchDev* dev) {
    // The batch table is larger than a kernel argument: copy the used prefix of each array.
    cudaMemcpyAsync(dev, &host, sizeof(FxBatchDev), cudaMemcpyHostToDevice, s);
}

void fx_launch_check_div(cudaStream_t s, float d, float rcp, float lo, float hi, unsigned long long* mismatches) {
    fxk_check_div<<<num_sms() * 16, 256, 0, s>>>(d, rcp, lo, hi, mismatches);
}
