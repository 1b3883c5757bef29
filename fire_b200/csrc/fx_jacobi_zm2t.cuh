// fx_jacobi_zm2t.cuh — the two-sweep Jacobi pass of fx_jacobi_zm2.cuh (solvePressureGlobal,
// shaders.ts:375-403, two sweeps per read of pressure and divergence) with its input planes
// staged by the Tensor Memory Accelerator instead of per-thread cp.async copies.
//
// Per plane, one elected thread issues two tiled tensor loads (cp.async.bulk.tensor.3d) into
// the plane's ring slot: the pressure box of 40 x 34 floats (x0 - 4 .. x0 + 35, y0 - 2 ..
// y0 + 31) and the divergence box of 40 x 32 floats (x0 - 4 .. x0 + 35, y0 - 1 .. y0 + 30),
// both completing on the slot's mbarrier (expect_tx of the boxes' bytes). Every thread waits
// on the slot's barrier phase before it reads the plane; a slot is refilled only after the
// step barrier that follows its last reads. The tensor maps cover this GPU's own buffers
// (the simulation's pressure pair, correction pair and divergence), loads only, no
// multicast: the code runs on one GPU. Box rows and columns outside the grid arrive as
// zeros (the tensor map's out-of-bound fill), so the clamped neighbour of row 0 is taken from
// the cell itself, as the single-sweep kernels take it; rows past the top are never read (the
// top row's update is 0), columns outside the grid never either (the x clamps use the cell).
//
// The arithmetic, the tile, the rings and the order of the two sweeps are those of
// fx_jacobi_zm2.cuh, so the results are bit-identical to it and to single sweeps. FP32
// pressure only: the tensor map's row stride must be a multiple of 16 bytes, which FP16 rows
// are only when X is a multiple of 8 (508 is not); FP16 pressure keeps the cp.async staging.
//
// The barrier waits are bounded (FX_T2_WAIT_LIMIT polls of try_wait): on expiry the CTA sets
// the simulation's error word, waits (bounded again) for its loads in flight and returns.
#pragma once

#include <cuda.h>

#include "fx_async.cuh"
#include "fx_jacobi_zm2.cuh"

#ifndef FX_T2_SLOTS
#define FX_T2_SLOTS 6
#endif
#define FX_T2_AHEAD (FX_T2_SLOTS - 3)  // step z issues the loads of plane z + AHEAD
#define FX_T2_PBOX_Y FX_Z2_PROWS       // 34 rows of 40 floats
#define FX_T2_DBOX_Y FX_Z2_RROWS       // 32 rows of 40 floats
#define FX_T2_PBYTES (FX_Z2_COLS * FX_T2_PBOX_Y * 4)  // 5440
#define FX_T2_DBYTES (FX_Z2_COLS * FX_T2_DBOX_Y * 4)  // 5120
#define FX_T2_PSLOT 1376                // floats per pressure slot: 5440 B padded to 43 x 128 B
#define FX_T2_DSLOT (FX_Z2_COLS * FX_T2_DBOX_Y)  // 1280 floats = 40 x 128 B
#define FX_T2_WAIT_LIMIT (1u << 22)
#ifndef FX_T2_ONE_WAITER
#define FX_T2_ONE_WAITER 1
#endif
#ifndef FX_T2_ISSUE_EARLY  // issue a plane's loads right after the step barrier (else at its end)
#define FX_T2_ISSUE_EARLY 1
#endif

// Tensor maps of a simulation (FxSimDev::tmap): pressure pair, correction pair, divergence.
enum { FX_TM_P0 = 0, FX_TM_P1 = 1, FX_TM_C0 = 2, FX_TM_C1 = 3, FX_TM_DIV = 4, FX_TM_COUNT = 5 };

struct FxT2Smem {
    alignas(128) float p[FX_T2_SLOTS][FX_T2_PSLOT];
    alignas(128) float d[FX_T2_SLOTS][FX_T2_DSLOT];
    alignas(128) float s[FX_Z2_SSLOTS][FX_Z2_RROWS * FX_Z2_COLS];
    alignas(8) unsigned long long bar[FX_T2_SLOTS];
    int err;
};
static_assert(FX_T2_PSLOT * 4 >= FX_T2_PBYTES && (FX_T2_PSLOT * 4) % 128 == 0, "pressure slots: 128-byte aligned");
static_assert((FX_T2_DSLOT * 4) % 128 == 0, "divergence slots: 128-byte aligned");

// A 3-D tiled tensor load of the box at (x, y, z) into shared memory, completing on bar.
FXD void fx_tma_load3(void* dst, const CUtensorMap* map, int x, int y, int z, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(fx_smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(fx_smem_u32(bar))
        : "memory");
}

// Makes the tensor map at `map` (written by the host before the launch) visible to the TMA
// unit's proxy before this CTA's first load through it.
FXD void fx_tmap_acquire(const CUtensorMap* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(reinterpret_cast<unsigned long long>(map))
                 : "memory");
}

// The tensor map of the solve's input buffer.
FXD const CUtensorMap* fx_t2_map_of(const FxSimDev& S, const void* buf) {
    const int i = buf == S.p[0] ? FX_TM_P0 : (buf == S.p[1] ? FX_TM_P1 : (buf == S.corr[0] ? FX_TM_C0 : FX_TM_C1));
    return &S.tmap[i];
}

// Two sweeps of one tile column: planes [z0, z1) of tile (x0, y0); pin (its map tmP) ->
// pout. `phases` holds the parity of each slot's next barrier phase (bit per slot). False
// when a barrier wait ran out (the error word is set and no load of this CTA is in flight).
template <bool ZERO_IN>
FXD bool fx_zm2t_tile(const FxSimDev& S, const CUtensorMap* tmP, float* __restrict__ pout, int x0, int y0, int z0,
                      int z1, FxT2Smem& sm, unsigned& phases) {
    const int X = S.X, Y = S.Y, Z = S.Z;
    const long long XY = (long long)X * Y;
    const FxJacobiConst2 c2 = fx_jacobi_const2(FxJacobiConst{S.jc[0], S.jc[1], S.jc[2], S.jc[3]}, S.jcRcp, S.jcFastDiv != 0);
    const CUtensorMap* tmD = &S.tmap[FX_TM_DIV];
    const int t = threadIdx.x, cg = t & 7, row = t >> 3;
    const int x = x0 + 4 * cg, y = y0 - 1 + row;
    const bool in1 = x < X && y >= 0 && y < Y;
    const bool in2 = in1 && row >= 1 && row <= FX_Z2_TY;
    const int cj = t - 192, cside = cj >= FX_Z2_TY ? 1 : 0, cr = cj - cside * FX_Z2_TY;
    const int cx = cside ? x0 + FX_Z2_TX : x0 - 1, cy = y0 + cr;
    const bool hCol = t >= 192 && t < 192 + 2 * FX_Z2_TY && cx >= 0 && cx < X && cy < Y;

    const int zs1 = max(z0 - 1, 0), ze1 = min(z1, Z - 1);  // sweep-1 planes of this chunk
    const int qa = zs1 - 1, qb = ze1 + 1;                  // input planes (clamped into the grid)
    auto p4 = [&](int slot, int r, int col) {
        return ZERO_IN ? make_float4(0, 0, 0, 0) : *reinterpret_cast<const float4*>(&sm.p[slot][r * FX_Z2_COLS + col]);
    };
    auto p1 = [&](int slot, int r, int col) { return ZERO_IN ? 0.0f : sm.p[slot][r * FX_Z2_COLS + col]; };
    const int pcol = 4 + 4 * cg, prow = row + 1, o0 = row * FX_Z2_COLS + pcol;
    const unsigned bytes = (ZERO_IN ? 0u : (unsigned)FX_T2_PBYTES) + (unsigned)FX_T2_DBYTES;
    auto issue = [&](int q, int slot) {  // thread 0 only
        const int qc = q < 0 ? 0 : (q > Z - 1 ? Z - 1 : q);
        fx_mbar_expect_tx(&sm.bar[slot], bytes);
        if (!ZERO_IN) fx_tma_load3(sm.p[slot], tmP, x0 - 4, y0 - 2, qc, &sm.bar[slot]);
        fx_tma_load3(sm.d[slot], tmD, x0 - 4, y0 - 1, qc, &sm.bar[slot]);
    };
    // waits for the plane in `slot`; on expiry every thread learns it at the next barrier.
    // With FX_T2_ONE_WAITER one thread polls the barrier and the step's CTA barrier that
    // follows passes the landed plane on to the others (the TMA writes the waiting thread
    // observed are ordered before everything after the CTA barrier); else every thread polls.
    auto wait = [&](int slot) {
        if (!FX_T2_ONE_WAITER || t == 0)
            if (!fx_mbar_wait(&sm.bar[slot], (phases >> slot) & 1u, FX_T2_WAIT_LIMIT)) sm.err = 1;
        phases ^= 1u << slot;
    };
    if (t == 0) {
        fx_tmap_acquire(tmD);
        if (!ZERO_IN) fx_tmap_acquire(tmP);
        for (int q = qa; q <= min(qa + FX_T2_AHEAD, qb); ++q) issue(q, q - qa);
    }
    int issued = min(qa + FX_T2_AHEAD, qb);  // last plane issued (uniform over the CTA)
    int waited = qa - 1;                     // last plane waited for
    // slot of plane q: (q - qa) mod SLOTS; s0 tracks plane z's slot incrementally
    int s0 = 1;
    for (int z = zs1; z <= ze1 + 2; ++z) {
        const int sm1 = s0 == 0 ? FX_T2_SLOTS - 1 : s0 - 1, sp1 = s0 == FX_T2_SLOTS - 1 ? 0 : s0 + 1;
        for (int q = waited + 1; q <= min(z + 1, issued); ++q) wait((q - qa) % FX_T2_SLOTS);
        waited = max(waited, min(z + 1, issued));
        __syncthreads();  // planes up to z + 1 landed for every thread; sweep-1 plane z - 1 is
                          // complete, and step z - 1's reads of the slot of plane z - 3 are done
        if (sm.err) break;
        const int qn = z + FX_T2_AHEAD;  // into the slot of plane z - 3, read last in step z - 1
        if (FX_T2_ISSUE_EARLY && qn <= qb) {
            if (t == 0) issue(qn, (qn - qa) % FX_T2_SLOTS);
            issued = qn;
        }
        // ---- sweep 2 on plane z - 2 (from the sweep-1 ring)
        {
            const int qz = z - 2;
            const bool do2 = qz >= z0 && qz < z1;
            const float* s2 = sm.s[qz & (FX_Z2_SSLOTS - 1)];
            const float4 cen2 = do2 && in2 ? *reinterpret_cast<const float4*>(s2 + o0) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const float fromL2 = __shfl_up_sync(0xffffffffu, cen2.w, 1), fromR2 = __shfl_down_sync(0xffffffffu, cen2.x, 1);
            if (do2 && in2) {
                float4 o = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (y != Y - 1) {
                    const float* sk = qz > 0 ? sm.s[(qz - 1) & (FX_Z2_SSLOTS - 1)] : s2;
                    const float* sf = qz < Z - 1 ? sm.s[(qz + 1) & (FX_Z2_SSLOTS - 1)] : s2;
                    const float l = x == 0 ? cen2.x : (cg > 0 ? fromL2 : s2[o0 - 1]);
                    const float rr = x + 3 == X - 1 ? cen2.w : (cg < 7 ? fromR2 : s2[o0 + 4]);
                    const float4 b = y > 0 ? *reinterpret_cast<const float4*>(s2 + o0 - FX_Z2_COLS) : cen2;
                    const float4 tt = *reinterpret_cast<const float4*>(s2 + o0 + FX_Z2_COLS);
                    const float4 dv =
                        *reinterpret_cast<const float4*>(&sm.d[s0 >= 2 ? s0 - 2 : s0 + FX_T2_SLOTS - 2][o0]);
                    o = fx_jacobi4(c2, l, cen2, rr, b, tt, *reinterpret_cast<const float4*>(sk + o0),
                                   *reinterpret_cast<const float4*>(sf + o0), dv);
                }
                PStore<float>::st4(pout, (long long)qz * XY + (long long)y * X + x, o);
            }
        }
        // ---- sweep 1 on plane z over the tile and its ring
        if (z <= ze1) {
            float* out = sm.s[z & (FX_Z2_SSLOTS - 1)];
            const float4 cen = in1 ? p4(s0, prow, pcol) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            const float fromL = __shfl_up_sync(0xffffffffu, cen.w, 1), fromR = __shfl_down_sync(0xffffffffu, cen.x, 1);
            if (in1) {
                float4 o = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (y != Y - 1) {
                    const float l = x == 0 ? cen.x : (cg > 0 ? fromL : p1(s0, prow, pcol - 1));
                    const float rr = x + 3 == X - 1 ? cen.w : (cg < 7 ? fromR : p1(s0, prow, pcol + 4));
                    const float4 dv = *reinterpret_cast<const float4*>(&sm.d[s0][o0]);
                    const float4 b = y > 0 ? p4(s0, prow - 1, pcol) : cen;  // row -1 arrives as zeros
                    o = fx_jacobi4(c2, l, cen, rr, b, p4(s0, prow + 1, pcol), p4(sm1, prow, pcol), p4(sp1, prow, pcol),
                                   dv);
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
                    const float b = cy > 0 ? p1(s0, hrow - 1, hcol) : c;
                    o = fx_jacobi1(c2, l, rr, b, p1(s0, hrow + 1, hcol), p1(sm1, hrow, hcol), p1(sp1, hrow, hcol),
                                   sm.d[s0][srow * FX_Z2_COLS + hcol]);
                }
                out[srow * FX_Z2_COLS + hcol] = o;
            }
        }
        if (!FX_T2_ISSUE_EARLY && qn <= qb) {  // the loads of plane z + AHEAD at the step's end
            if (t == 0) issue(qn, (qn - qa) % FX_T2_SLOTS);
            issued = qn;
        }
        s0 = sp1;
    }
    __syncthreads();  // every thread's waits of this tile are done; sm.err is final
    if (sm.err) {
        // drain the loads still in flight (bounded), so none lands after the CTA returns
        if (t == 0) {
            for (int q = waited + 1; q <= issued; ++q) {
                const int slot = (q - qa) % FX_T2_SLOTS;
                fx_mbar_wait(&sm.bar[slot], (phases >> slot) & 1u, FX_T2_WAIT_LIMIT);
                phases ^= 1u << slot;
            }
        }
        return false;
    }
    return true;
}
