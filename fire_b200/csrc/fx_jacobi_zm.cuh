// fx_jacobi_zm.cuh — one Jacobi sweep (solvePressureGlobal, shaders.ts:375-403) by
// z-marching tiles with an asynchronous shared-memory pipeline.
//
// A CTA of 256 threads owns an x-y tile of 128 x 8 cells (lane: 4 consecutive x cells,
// warp: one row) and walks a chunk of z planes. Pressure planes, with a one-row halo
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
#define FX_ZM_TX 128  // tile cells in x (32 lanes x 4)
#define FX_ZM_TY 8    // tile rows in y (8 warps)
#define FX_ZM_SLOTS 6
#define FX_ZM_COLS (FX_ZM_TX + 8)  // 4-cell halo segment on each side
#define FX_ZM_ROWS (FX_ZM_TY + 2)

__host__ __device__ inline int fx_zm_bricks(int X, int Y, int Z, int zc) {
    return ((X + FX_ZM_TX - 1) / FX_ZM_TX) * ((Y + FX_ZM_TY - 1) / FX_ZM_TY) * ((Z + zc - 1) / zc);
}

template <typename PT>
struct FxZmSmem {
    PT p[FX_ZM_SLOTS][FX_ZM_ROWS][FX_ZM_COLS];
    float d[FX_ZM_SLOTS][FX_ZM_TY][FX_ZM_TX];
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

// Issues the copies of plane q (clamped) into ring slot `slot`: the tile rows, the halo
// rows and the halo segments (pressure), and the tile rows of the divergence when
// withDiv (the plane is one the chunk updates).
template <typename PT>
FXD void fx_zm_issue(FxZmSmem<PT>& sm, int slot, const PT* __restrict__ p, const float* __restrict__ div, int X, int Y,
                     int Z, int x0t, int y0t, int q, bool loadP, bool withDiv) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int qc = q < 0 ? 0 : (q > Z - 1 ? Z - 1 : q);
    const long long plane = (long long)qc * X * Y;
    const int x = x0t + 4 * lane;
    if (loadP) {
        // rows: warp w loads tile row w and, for w < 2, one halo row (w = 0: below, 1: above)
        for (int r = w; r < FX_ZM_ROWS; r += 8) {
            const int gy = y0t - 1 + r;
            const int cy = gy < 0 ? 0 : (gy > Y - 1 ? Y - 1 : gy);
            const PT* row = p + plane + (long long)cy * X;
            if (x < X) fx_cp4(&sm.p[slot][r][4 + 4 * lane], row + x);
            if (r >= 1 && r <= FX_ZM_TY) {  // halo segments of the tile rows
                if (lane == 0 && x0t >= 4) fx_cp4(&sm.p[slot][r][0], row + x0t - 4);
                if (lane == 31 && x0t + FX_ZM_TX < X) fx_cp4(&sm.p[slot][r][4 + FX_ZM_TX], row + x0t + FX_ZM_TX);
            }
        }
    }
    if (withDiv) {
        const int gy = y0t + w;
        if (x < X && gy < Y) fx_cp_async16(&sm.d[slot][w][4 * lane], div + plane + (long long)gy * X + x);
    }
}

// Four consecutive shared-memory pressure elements as float4 (one 16- or 8-byte read).
FXD float4 fx_zm_ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
FXD float4 fx_zm_ld4(const __half* p) {
    const uint2 r = *reinterpret_cast<const uint2*>(p);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&r.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&r.y));
    return make_float4(a.x, a.y, b.x, b.y);
}

// One z-marching tile of one sweep: planes [z0, z1) of the tile (x0t, y0t). ZERO_IN: the
// input is known to be zero (the first sweep of a cleared solve): no pressure loads.
template <typename PT, bool ZERO_IN>
FXD void fx_zm_tile(const FxSimDev* __restrict__ Sp, const PT* __restrict__ pin, PT* __restrict__ pout, int x0t, int y0t,
                    int z0, int z1, FxZmSmem<PT>& sm) {
    const FxSimDev& S = *Sp;
    const int X = S.X, Y = S.Y, Z = S.Z;
    const float* __restrict__ div = S.div;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int x = x0t + 4 * lane, y = y0t + w;
    const bool active = x < X && y < Y;
    const FxJacobiConst c{S.jc[0], S.jc[1], S.jc[2], S.jc[3]};
    const float rcpD = S.jcRcp;
    const bool fastDiv = S.jcFastDiv != 0;
    constexpr bool loadP = !ZERO_IN;
    // ring: at plane z, slots hold z-1, z, z+1 (read), z+2, z+3 (in flight) and the
    // slot of z-2, refilled with z+4 right after the barrier
    // prologue: planes z0-1 .. z0+3 (pressure), divergence for those in [z0, z1)
    for (int q = z0 - 1; q <= z0 + 3; ++q) {
        fx_zm_issue<PT>(sm, (q + FX_ZM_SLOTS) % FX_ZM_SLOTS, pin, div, X, Y, Z, x0t, y0t, q, loadP, q >= z0 && q < z1);
        fx_cp_commit();
    }
    for (int z = z0; z < z1; ++z) {
        fx_cp_wait<2>();  // this thread's copies of planes up to z + 1 have landed
        __syncthreads();  // ... everyone's; and everyone is done with plane z - 2
        {
            const int q = z + 4;
            fx_zm_issue<PT>(sm, (q + FX_ZM_SLOTS) % FX_ZM_SLOTS, pin, div, X, Y, Z, x0t, y0t, q, loadP && q <= z1, q < z1);
            fx_cp_commit();
        }
        const int sm1 = (z - 1 + FX_ZM_SLOTS) % FX_ZM_SLOTS, s0 = z % FX_ZM_SLOTS, sp1 = (z + 1) % FX_ZM_SLOTS;
        if (active) {
            float4 out;
            if (y == Y - 1) {
                out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // the open top is the ambient boundary
            } else {
                const int r = w + 1, col = 4 + 4 * lane;
                const float4 dv = *reinterpret_cast<const float4*>(&sm.d[s0][w][4 * lane]);
                float4 cen = make_float4(0, 0, 0, 0), b = cen, t = cen, k = cen, f = cen;
                float l = 0.0f, rr = 0.0f;
                if (loadP) {
                    cen = fx_zm_ld4(&sm.p[s0][r][col]);
                    b = fx_zm_ld4(&sm.p[s0][r - 1][col]);
                    t = fx_zm_ld4(&sm.p[s0][r + 1][col]);
                    k = fx_zm_ld4(&sm.p[sm1][r][col]);
                    f = fx_zm_ld4(&sm.p[sp1][r][col]);
                    l = x == 0 ? cen.x : (float)sm.p[s0][r][col - 1];
                    rr = x + 3 == X - 1 ? cen.w : (float)sm.p[s0][r][col + 4];
                }
                float o[4];
                o[0] = fx_jacobi_numerator(c, l, cen.y, b.x, t.x, k.x, f.x, dv.x);
                o[1] = fx_jacobi_numerator(c, cen.x, cen.z, b.y, t.y, k.y, f.y, dv.y);
                o[2] = fx_jacobi_numerator(c, cen.y, cen.w, b.z, t.z, k.z, f.z, dv.z);
                o[3] = fx_jacobi_numerator(c, cen.z, rr, b.w, t.w, k.w, f.w, dv.w);
#pragma unroll
                for (int i = 0; i < 4; ++i) o[i] = fastDiv ? fx_div_by_const(o[i], c.denom, rcpD) : __fdiv_rn(o[i], c.denom);
                out = make_float4(o[0], o[1], o[2], o[3]);
            }
            PStore<PT>::st4(pout, (long long)z * X * Y + (long long)y * X + x, out);
        }
    }
    fx_cp_wait<0>();
    __syncthreads();
}
