// fx_jacobi_zm2.cuh — two Jacobi sweeps (solvePressureGlobal, shaders.ts:375-403) per pass
// over HBM: the z-marching tile of fx_jacobi_zm.cuh widened by a one-cell ring, with the
// first sweep's values kept in shared memory for the second.
//
// A CTA owns a 32 x 30 tile of x-y and a chunk of z planes. It streams input pressure
// planes (tile plus two rows and one 4-cell segment on each side) and divergence planes
// (tile plus one row and one segment) through cp.async rings, as the single-sweep kernel
// does. At step z it computes sweep 2 on plane z - 2 over the tile from sweep-1 planes
// z - 3 .. z - 1 and stores it, then sweep 1 on plane z over the tile and its one-cell ring
// into a ring of sweep-1 planes: the 32 rows y0 - 1 .. y0 + 30 as 4-cell groups, one per
// thread (256 threads, 8 groups a row: every warp does the same work), and the ring's two
// columns cell by cell (60 cells, on the last two warps). Both finish before the step's
// barrier, so one barrier per step orders everything. Sweep 2 is the only value stored. The chunk's sweep-1 planes reach one plane past
// it at each end, so each chunk is independent.
//
// Every update is the single sweep's FP32 computation (fx_jacobi4, or fx_jacobi1 for
// single ring cells: both give the IEEE quotient), the open top row is 0 after each
// sweep, and with FP16 storage the sweep-1 values are rounded to FP16 as a stored sweep
// would be: two fused sweeps are bit-identical to two single sweeps. Boundaries follow the
// reference's clamped addressing: input rows and planes are loaded clamped into the grid,
// so sweep 1 sees its clamped neighbours; sweep 2 takes a neighbour that the clamp maps
// onto the cell itself from the cell.
#pragma once

#include "fx_jacobi_zm.cuh"
#include "fx_step_math.cuh"
#include "fx_storage.cuh"

#define FX_Z2_THREADS 256
#define FX_Z2_TX 32          // tile width (8 groups of 4 cells)
#define FX_Z2_TY 30          // tile height: with its ring rows, one group row per thread row
#define FX_Z2_COLS 40        // slot row: 4-cell segment, 32 cells, 4-cell segment
#define FX_Z2_PROWS 34       // input pressure rows: y0 - 2 .. y0 + 31
#define FX_Z2_RROWS 32       // divergence and sweep-1 rows: y0 - 1 .. y0 + 30
#ifndef FX_Z2_SLOTS
#define FX_Z2_SLOTS 6        // input and divergence rings: planes z - 2 .. z + SLOTS - 3 at step z
#endif
#define FX_Z2_AHEAD (FX_Z2_SLOTS - 3)  // step z issues the copies of plane z + AHEAD
static_assert(FX_Z2_SLOTS >= 5, "planes z - 2 .. z + 2 must fit the rings");
#ifndef FX_Z2_MINB
#define FX_Z2_MINB 2         // CTAs per SM the registers are budgeted for
#endif
#define FX_Z2_SSLOTS 4       // sweep-1 ring: planes z - 3 .. z - 1 (read) and z (written)

template <typename PT>
struct FxZ2Smem {
    PT p[FX_Z2_SLOTS][FX_Z2_PROWS * FX_Z2_COLS];
    float d[FX_Z2_SLOTS][FX_Z2_RROWS * FX_Z2_COLS];
    float s[FX_Z2_SSLOTS][FX_Z2_RROWS * FX_Z2_COLS];
};

// Bricks (tile x tile x z chunk) of one grid.
__host__ __device__ inline int fx_zm2_bricks(int X, int Y, int Z, int zc) {
    return ((X + FX_Z2_TX - 1) / FX_Z2_TX) * ((Y + FX_Z2_TY - 1) / FX_Z2_TY) * ((Z + zc - 1) / zc);
}

// This thread's copies of one plane: up to two input segments and two divergence segments
// (offsets within a plane and within a slot; -1: none).
struct FxZ2Plan {
    int gP[2], sP[2], gD[2], sD[2];
};
FXD FxZ2Plan fx_zm2_plan(int X, int Y, int x0, int y0) {
    FxZ2Plan P;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int i = threadIdx.x + k * FX_Z2_THREADS;
        P.gP[k] = P.sP[k] = P.gD[k] = P.sD[k] = -1;
        if (i < FX_Z2_PROWS * 10) {
            const int row = i / 10, seg = i - row * 10;
            const int gx = x0 - 4 + 4 * seg;
            const int gy = y0 - 2 + row, cy = gy < 0 ? 0 : (gy > Y - 1 ? Y - 1 : gy);
            if (gx >= 0 && gx < X) {
                P.gP[k] = cy * X + gx;
                P.sP[k] = row * FX_Z2_COLS + 4 * seg;
            }
        }
        if (i < FX_Z2_RROWS * 10) {
            const int row = i / 10, seg = i - row * 10;
            const int gx = x0 - 4 + 4 * seg, gy = y0 - 1 + row;
            if (gx >= 0 && gx < X && gy >= 0 && gy < Y) {
                P.gD[k] = gy * X + gx;
                P.sD[k] = row * FX_Z2_COLS + 4 * seg;
            }
        }
    }
    return P;
}

template <typename PT>
FXD void fx_zm2_issue(FxZ2Smem<PT>& sm, const FxZ2Plan& P, const PT* __restrict__ p, const float* __restrict__ div,
                      long long XY, int Z, int q, int slot, bool loadP, bool withDiv) {
    const int qc = q < 0 ? 0 : (q > Z - 1 ? Z - 1 : q);
    const long long plane = (long long)qc * XY;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        if (loadP && P.sP[k] >= 0) fx_cp4(&sm.p[slot][P.sP[k]], p + plane + P.gP[k]);
        if (withDiv && P.sD[k] >= 0) fx_cp_async16(&sm.d[slot][P.sD[k]], div + plane + P.gD[k]);
    }
}

template <bool ROUND>
FXD float4 fx_z2_round(float4 o) {
    if (ROUND) o = make_float4(PStore<__half>::round(o.x), PStore<__half>::round(o.y), PStore<__half>::round(o.z),
                               PStore<__half>::round(o.w));
    return o;
}

// Two sweeps of one tile column: planes [z0, z1) of tile (x0, y0); pin -> pout.
template <typename PT, bool ZERO_IN, bool ROUND>
FXD void fx_zm2_tile(const FxSimDev& S, const PT* __restrict__ pin, PT* __restrict__ pout, int x0, int y0, int z0, int z1,
                     FxZ2Smem<PT>& sm) {
    const int X = S.X, Y = S.Y, Z = S.Z;
    const long long XY = (long long)X * Y;
    const float* __restrict__ div = S.div;
    const FxJacobiConst2 c2 = fx_jacobi_const2(FxJacobiConst{S.jc[0], S.jc[1], S.jc[2], S.jc[3]}, S.jcRcp, S.jcFastDiv != 0);
    // this thread's group: 4 cells at (x0 + 4 cg, y0 - 1 + row); sweep-1 row `row` of the
    // ring, and for rows 1..30 the tile's row row - 1 in sweep 2
    const int t = threadIdx.x, cg = t & 7, row = t >> 3;
    const int x = x0 + 4 * cg, y = y0 - 1 + row;
    const bool in1 = x < X && y >= 0 && y < Y;               // sweep 1 on this group
    const bool in2 = in1 && row >= 1 && row <= FX_Z2_TY;     // sweep 2 on this group
    constexpr bool loadP = !ZERO_IN;
    const FxZ2Plan plan = fx_zm2_plan(X, Y, x0, y0);
    // ring columns x0 - 1 and x0 + 32, rows y0 .. y0 + 29: one cell each on threads 192-251
    const int cj = t - 192, cside = cj >= FX_Z2_TY ? 1 : 0, cr = cj - cside * FX_Z2_TY;
    const int cx = cside ? x0 + FX_Z2_TX : x0 - 1, cy = y0 + cr;
    const bool hCol = t >= 192 && t < 192 + 2 * FX_Z2_TY && cx >= 0 && cx < X && cy < Y;

    const int zs1 = max(z0 - 1, 0), ze1 = min(z1, Z - 1);  // sweep-1 planes of this chunk
    auto p4 = [&](int slot, int r, int col) { return loadP ? fx_zm_ld4(&sm.p[slot][r * FX_Z2_COLS + col]) : make_float4(0, 0, 0, 0); };
    auto p1 = [&](int slot, int r, int col) { return loadP ? (float)sm.p[slot][r * FX_Z2_COLS + col] : 0.0f; };
    const int pcol = 4 + 4 * cg;           // the group's column in every slot
    const int prow = row + 1;              // its input row (input rows start at y0 - 2)
    const int o0 = row * FX_Z2_COLS + pcol;  // its offset in divergence and sweep-1 slots

    // ring slots: plane q lives in slot q mod 7 of the input and divergence rings and in
    // slot q mod 4 (q & 3, q >= -2) of the sweep-1 ring; s0 tracks z mod 7 incrementally
    int s0 = zs1 % FX_Z2_SLOTS;
    for (int q = zs1 - 1; q <= zs1 + FX_Z2_AHEAD - 1; ++q) {
        fx_zm2_issue<PT>(sm, plan, pin, div, XY, Z, q, (q + FX_Z2_SLOTS) % FX_Z2_SLOTS, loadP, q >= zs1 && q <= ze1);
        fx_cp_commit();
    }
    for (int z = zs1; z <= ze1 + 2; ++z) {
        const int sm1 = s0 == 0 ? FX_Z2_SLOTS - 1 : s0 - 1, sp1 = s0 == FX_Z2_SLOTS - 1 ? 0 : s0 + 1;
        fx_cp_wait<FX_Z2_AHEAD - 2>();  // this thread's copies of planes up to z + 1 have landed
        __syncthreads();  // ... everyone's; sweep-1 plane z - 1 is complete, and so are step
                          // z - 1's reads of plane z - 3, whose slots are refilled at the end
        auto sweep1 = [&]() {
            if (z <= ze1) {  // ---- sweep 1 on plane z
                float* out = sm.s[z & (FX_Z2_SSLOTS - 1)];
                // x neighbours from the adjacent lanes (the same row's groups cg - 1, cg + 1); the
                // row's end groups read the ring segments
                const float4 cen = in1 ? p4(s0, prow, pcol) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                const float fromL = __shfl_up_sync(0xffffffffu, cen.w, 1), fromR = __shfl_down_sync(0xffffffffu, cen.x, 1);
                if (in1) {
                    float4 o = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    if (y != Y - 1) {
                        const float l = x == 0 ? cen.x : (cg > 0 ? fromL : p1(s0, prow, pcol - 1));
                        const float rr = x + 3 == X - 1 ? cen.w : (cg < 7 ? fromR : p1(s0, prow, pcol + 4));
                        const float4 dv = *reinterpret_cast<const float4*>(&sm.d[s0][o0]);
                        o = fx_jacobi4(c2, l, cen, rr, p4(s0, prow - 1, pcol), p4(s0, prow + 1, pcol), p4(sm1, prow, pcol),
                                       p4(sp1, prow, pcol), dv);
                        o = fx_z2_round<ROUND>(o);
                    }
                    *reinterpret_cast<float4*>(&out[o0]) = o;
                }
                if (hCol) {
                    const int hrow = cr + 2, hcol = cx - (x0 - 4), srow = cr + 1;
                    float o = 0.0f;
                    if (cy != Y - 1) {
                        const float c = p1(s0, hrow, hcol);
                        const float l = cx == 0 ? c : p1(s0, hrow, hcol - 1);
                        const float rr = cx == X - 1 ? c : p1(s0, hrow, hcol + 1);
                        o = fx_jacobi1(c2, l, rr, p1(s0, hrow - 1, hcol), p1(s0, hrow + 1, hcol), p1(sm1, hrow, hcol),
                                       p1(sp1, hrow, hcol), sm.d[s0][srow * FX_Z2_COLS + hcol]);
                        if (ROUND) o = PStore<__half>::round(o);
                    }
                    out[srow * FX_Z2_COLS + hcol] = o;
                }
            }
        };
        auto sweep2 = [&]() {
            const int qz = z - 2;  // ---- sweep 2 on plane z - 2
            const bool do2 = qz >= z0 && qz < z1;  // uniform over the CTA
            const float* s2 = sm.s[qz & (FX_Z2_SSLOTS - 1)];
            const float4 cen2 = do2 && in2 ? *reinterpret_cast<const float4*>(s2 + o0) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const float fromL2 = __shfl_up_sync(0xffffffffu, cen2.w, 1), fromR2 = __shfl_down_sync(0xffffffffu, cen2.x, 1);
            if (do2 && in2) {
                float4 o = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (y != Y - 1) {
                    const float* sk = qz > 0 ? sm.s[(qz - 1) & (FX_Z2_SSLOTS - 1)] : s2;
                    const float* sf = qz < Z - 1 ? sm.s[(qz + 1) & (FX_Z2_SSLOTS - 1)] : s2;
                    const float4 cen = cen2;
                    const float l = x == 0 ? cen.x : (cg > 0 ? fromL2 : s2[o0 - 1]);
                    const float rr = x + 3 == X - 1 ? cen.w : (cg < 7 ? fromR2 : s2[o0 + 4]);
                    const float4 b = y > 0 ? *reinterpret_cast<const float4*>(s2 + o0 - FX_Z2_COLS) : cen;
                    const float4 tt = *reinterpret_cast<const float4*>(s2 + o0 + FX_Z2_COLS);
                    // divergence plane z - 2: slot (z - 2) mod 7
                    const float4 dv = *reinterpret_cast<const float4*>(&sm.d[s0 >= 2 ? s0 - 2 : s0 + FX_Z2_SLOTS - 2][o0]);
                    o = fx_jacobi4(c2, l, cen, rr, b, tt, *reinterpret_cast<const float4*>(sk + o0),
                                   *reinterpret_cast<const float4*>(sf + o0), dv);
                }
                PStore<PT>::st4(pout, (long long)qz * XY + (long long)y * X + x, o);
            }
        };
        // sweep 2 first: its global stores drain while sweep 1 computes; the copies of plane
        // z + AHEAD last, after both sweeps' shared-memory loads (measured: 49.6 ms of Jacobi
        // per 508^3 step with sweep 1 first and the copies right after the barrier, 47.7 with
        // sweep 2 first, 45.2 with the copies here)
        sweep2();
        sweep1();
        {
            const int q = z + FX_Z2_AHEAD;  // into the slots of plane z - 3: step z reads none
            fx_zm2_issue<PT>(sm, plan, pin, div, XY, Z, q, s0 >= 3 ? s0 - 3 : s0 + FX_Z2_AHEAD, loadP && q <= ze1 + 1, q <= ze1);
            fx_cp_commit();
        }
        s0 = sp1;
    }
    fx_cp_wait<0>();
    __syncthreads();
}
