// fx_jacobi_zm.cuh — one Jacobi sweep (solvePressureGlobal, shaders.ts:375-403) by
// z-marching tiles with an asynchronous shared-memory pipeline.
//
// A CTA of 256 threads owns an x-y tile of 1024 cells, 128 x 8, 64 x 16 or 32 x 32 (the
// widest that wastes the fewest lanes on the simulation's X; a thread takes 4
// consecutive x cells of one row) and walks a chunk of z planes. Pressure planes, with a one-row halo
// above and below and a 4-cell halo segment left and right, and the divergence rows
// stream into a ring of FX_ZM_SLOTS shared-memory slots through cp.async (16- or
// 8-byte global->shared copies that need no registers), three planes ahead of the plane
// being updated. Every neighbour of the update (x, y and z) is then read from shared
// memory, so each pressure value crosses L2 about once per sweep. One barrier per plane:
// the slot refilled at plane z held plane z - 2, which every thread finished reading
// before that barrier.
//
// Boundaries follow the reference: the halo rows are loaded from the clamped row (so the
// floor's lower neighbour is the floor itself), x neighbours at the walls select the cell
// itself, the z ends load the clamped plane, and the top row is written 0.
#pragma once

#include "fx_step_math.cuh"
#include "fx_storage.cuh"

#define FX_ZM_THREADS 256
#define FX_ZM_CELLS 1024  // tile cells per plane: TX x TY = 128 x 8, 64 x 16 or 32 x 32
#define FX_ZM_SLOTS 6
#define FX_ZM_PSLOT 1360  // pressure slot: (TY + 2) rows of (TX + 8) (largest of the three shapes)

// Tile width for an X-cell row: the widest of 128, 64, 32 that wastes the fewest lanes
// (X = 160 takes 32-wide tiles, X = 64 64-wide, X = 508 128-wide).
__host__ __device__ inline int fx_zm_tile_w(int X) {
    int best = 128, waste = ((X + 127) / 128) * 128 - X;
    for (int w = 64; w >= 32; w /= 2) {
        const int wst = ((X + w - 1) / w) * w - X;
        if (wst < waste) {
            best = w;
            waste = wst;
        }
    }
    return best;
}

__host__ __device__ inline int fx_zm_bricks(int X, int Y, int Z, int zc) {
    const int tx = fx_zm_tile_w(X), ty = FX_ZM_CELLS / tx;
    return ((X + tx - 1) / tx) * ((Y + ty - 1) / ty) * ((Z + zc - 1) / zc);
}

template <typename PT>
struct FxZmSmem {
    PT p[FX_ZM_SLOTS][FX_ZM_PSLOT];
    float d[FX_ZM_SLOTS][FX_ZM_CELLS];
};

FXD void fx_cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
FXD void fx_cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
FXD void fx_cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
FXD void fx_cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Copies 4 consecutive pressure elements (16 B of float, 8 B of half).
template <typename PT>
FXD void fx_cp4(PT* smem, const PT* gmem) {
    if (sizeof(PT) == 4) fx_cp_async16(smem, gmem);
    else fx_cp_async8(smem, gmem);
}

// Tile geometry of one thread: TX cells wide (L = TX / 4 lanes of 4 cells per row), TY
// rows; thread t takes row t / L and cell group t % L.
struct FxZmGeom {
    int tx, ty, cols;  // cols = TX + 8: a row with its 4-cell halo segments
    int cg, row;       // this thread's cell group and row
};
template <int TX>
FXD FxZmGeom fx_zm_geom() {
    FxZmGeom g;
    g.tx = TX;
    g.ty = FX_ZM_CELLS / TX;
    g.cols = TX + 8;
    g.cg = threadIdx.x % (TX / 4);
    g.row = threadIdx.x / (TX / 4);
    return g;
}

// This thread's share of the copies of one plane, fixed for the whole tile: offsets
// within a plane (global) and within a ring slot (shared); -1 marks a copy it does not
// make. Row r of a slot is tile-plus-halo row r (row 0 below the tile, row TY + 1 above,
// both clamped into the grid); thread row w copies row w and, for w < 2, row w + TY; the
// first and last cell groups of a row also copy its 4-cell halo segments.
struct FxZmPlan {
    int gP[2], sP[2];   // pressure row segments
    int gL, sL, gR, sR; // halo segments
    int gD, sD;         // divergence
};
FXD FxZmPlan fx_zm_plan(const FxZmGeom& G, int X, int Y, int x0t, int y0t) {
    FxZmPlan P;
    const int x = x0t + 4 * G.cg;
    const int L = G.tx >> 2;
    P.gL = P.sL = P.gR = P.sR = -1;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int r = G.row + k * G.ty;
        P.gP[k] = P.sP[k] = -1;
        if (r < G.ty + 2) {
            const int gy = y0t - 1 + r;
            const int cy = gy < 0 ? 0 : (gy > Y - 1 ? Y - 1 : gy);
            if (x < X) {
                P.gP[k] = cy * X + x;
                P.sP[k] = r * G.cols + 4 + 4 * G.cg;
            }
            if (r >= 1 && r <= G.ty) {
                if (G.cg == 0 && x0t >= 4) {
                    P.gL = cy * X + x0t - 4;
                    P.sL = r * G.cols;
                }
                if (G.cg == L - 1 && x0t + G.tx < X) {
                    P.gR = cy * X + x0t + G.tx;
                    P.sR = r * G.cols + 4 + G.tx;
                }
            }
        }
    }
    const int gy = y0t + G.row;
    P.gD = P.sD = -1;
    if (x < X && gy < Y) {
        P.gD = gy * X + x;
        P.sD = G.row * G.tx + 4 * G.cg;
    }
    return P;
}

// Issues this thread's copies of plane q (clamped into the grid) into ring slot `slot`:
// pressure when loadP, divergence when withDiv (the plane is one the chunk updates).
template <typename PT>
FXD void fx_zm_issue(FxZmSmem<PT>& sm, const FxZmPlan& P, int slot, const PT* __restrict__ p, const float* __restrict__ div,
                     long long XY, int Z, int q, bool loadP, bool withDiv) {
    const int qc = q < 0 ? 0 : (q > Z - 1 ? Z - 1 : q);
    const long long plane = (long long)qc * XY;
    if (loadP) {
        const PT* pp = p + plane;
        PT* sp = sm.p[slot];
        if (P.sP[0] >= 0) fx_cp4(sp + P.sP[0], pp + P.gP[0]);
        if (P.sP[1] >= 0) fx_cp4(sp + P.sP[1], pp + P.gP[1]);
        if (P.sL >= 0) fx_cp4(sp + P.sL, pp + P.gL);
        if (P.sR >= 0) fx_cp4(sp + P.sR, pp + P.gR);
    }
    if (withDiv && P.sD >= 0) fx_cp_async16(&sm.d[slot][P.sD], div + plane + P.gD);
}

// Four consecutive shared-memory pressure elements as float4 (one 16- or 8-byte read).
FXD float4 fx_zm_ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
FXD float4 fx_zm_ld4(const __half* p) {
    const uint2 r = *reinterpret_cast<const uint2*>(p);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&r.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&r.y));
    return make_float4(a.x, a.y, b.x, b.y);
}

// One z-marching tile of one sweep: planes [z0, z1) of the tile (x0t, y0t), TX cells wide.
// ZERO_IN: the input is known to be zero (the first sweep of a cleared solve): no
// pressure loads.
template <typename PT, bool ZERO_IN, int TX>
FXD void fx_zm_tile(const FxSimDev* __restrict__ Sp, const PT* __restrict__ pin, PT* __restrict__ pout, int x0t, int y0t,
                    int z0, int z1, FxZmSmem<PT>& sm) {
    const FxSimDev& S = *Sp;
    const int X = S.X, Y = S.Y, Z = S.Z;
    const float* __restrict__ div = S.div;
    const FxZmGeom G = fx_zm_geom<TX>();
    const int x = x0t + 4 * G.cg, y = y0t + G.row;
    const bool active = x < X && y < Y;
    const FxJacobiConst2 c2 = fx_jacobi_const2(FxJacobiConst{S.jc[0], S.jc[1], S.jc[2], S.jc[3]}, S.jcRcp, S.jcFastDiv != 0);
    constexpr bool loadP = !ZERO_IN;
    const FxZmPlan plan = fx_zm_plan(G, X, Y, x0t, y0t);
    const long long XY = (long long)X * Y;
    // ring: at plane z, slots hold z-1, z, z+1 (read), z+2, z+3 (in flight) and the
    // slot of z-2, refilled with z+4 right after the barrier
    // prologue: planes z0-1 .. z0+3 (pressure), divergence for those in [z0, z1)
    for (int q = z0 - 1; q <= z0 + 3; ++q) {
        fx_zm_issue<PT>(sm, plan, (q + FX_ZM_SLOTS) % FX_ZM_SLOTS, pin, div, XY, Z, q, loadP, q >= z0 && q < z1);
        fx_cp_commit();
    }
    const int r = G.row + 1, col = 4 + 4 * G.cg;
    for (int z = z0; z < z1; ++z) {
        fx_cp_wait<2>();  // this thread's copies of planes up to z + 1 have landed
        __syncthreads();  // ... everyone's; and everyone is done with plane z - 2
        {
            const int q = z + 4;
            fx_zm_issue<PT>(sm, plan, (q + FX_ZM_SLOTS) % FX_ZM_SLOTS, pin, div, XY, Z, q, loadP && q <= z1, q < z1);
            fx_cp_commit();
        }
        const int sm1 = (z - 1 + FX_ZM_SLOTS) % FX_ZM_SLOTS, s0 = z % FX_ZM_SLOTS, sp1 = (z + 1) % FX_ZM_SLOTS;
        if (active) {
            float4 out;
            if (y == Y - 1) {
                out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // the open top is the ambient boundary
            } else {
                const float4 dv = *reinterpret_cast<const float4*>(&sm.d[s0][G.row * G.tx + 4 * G.cg]);
                float4 cen = make_float4(0, 0, 0, 0), b = cen, t = cen, k = cen, f = cen;
                float l = 0.0f, rr = 0.0f;
                if (loadP) {
                    const PT* p0 = &sm.p[s0][r * G.cols + col];
                    cen = fx_zm_ld4(p0);
                    b = fx_zm_ld4(p0 - G.cols);
                    t = fx_zm_ld4(p0 + G.cols);
                    k = fx_zm_ld4(&sm.p[sm1][r * G.cols + col]);
                    f = fx_zm_ld4(&sm.p[sp1][r * G.cols + col]);
                    l = x == 0 ? cen.x : (float)p0[-1];
                    rr = x + 3 == X - 1 ? cen.w : (float)p0[4];
                }
                out = fx_jacobi4(c2, l, cen, rr, b, t, k, f, dv);
            }
            PStore<PT>::st4(pout, (long long)z * X * Y + (long long)y * X + x, out);
        }
    }
    fx_cp_wait<0>();
    __syncthreads();
}
