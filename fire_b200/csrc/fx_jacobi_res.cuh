// fx_jacobi_res.cuh — every sweep of one Jacobi phase (solvePressureGlobal,
// shaders.ts:375-403) in ONE cooperative launch, with the pressure resident on chip.
//
// Each simulation of the batch gets a group of CTAs (one per SM); CTA b of the group owns
// a box of by x bz rows (y, z) of full x rows and keeps the box's pressure, with a
// one-row halo on each side in y and z, and its divergence in shared memory for the
// whole phase. A sweep reads only shared memory: each thread computes its groups of 4
// consecutive x cells into registers, the CTA synchronises, then writes the new values
// back. Only box faces leave the SM: every sweep but the last computes the face groups
// first, stores them to the sweep's output buffer and publishes a per-box flag (release
// store), then computes the interior while the flag travels; after writing the new
// values back it waits for the flags of its up to four neighbours (acquire loads, bounded
// waits) and loads its halo rows from that buffer through L2 (ld.global.cg: L1 may hold
// stale lines). Only neighbours synchronise, so there is no
// group-wide barrier. A box rewrites a buffer two sweeps later, after its neighbours
// published the sweep in between, which they do only after reading that buffer's halo.
//
// Arithmetic, boundaries and buffer parity are those of one sweep per launch, so the
// result is bit-identical to the single-sweep kernels: the same numerator in the same
// order, the same division, FP16 rounding of every sweep's output when pressure is
// stored in FP16 (pressureShaders.ts:116), and the final values in the buffer that the
// reference's ping-pong would leave them in. The last two sweeps store every cell, so
// both buffers of the pair end as single sweeps leave them: the final result in one,
// the one before it in the other (the cold branch shares these buffers between the
// primary and residual solves, so the other buffer is observable there).
//
// A cooperative launch guarantees that every CTA is resident, so every neighbour flag
// arrives; the waits are still bounded (FX_RES_SPIN_LIMIT polls, or the simulation's own
// limit): on expiry the CTA sets the simulation's error word and returns, its neighbours'
// waits for it then expire in turn, every CTA returns, and the host reports a timeout.
#pragma once

#include "fx_async.cuh"
#include "fx_step_math.cuh"
#include "fx_storage.cuh"

#define FX_RES_THREADS 512
#define FX_RES_COPY_TC (FX_RES_THREADS - 32)  // compute threads of variant 4 (the last warp copies)
#define FX_RES_MAXG 12                // groups of 4 cells per thread, column variant
#define FX_RES_MAXF 4                 // face groups per thread, faces-first variant
#define FX_RES_MAXI 11                // interior groups per thread, faces-first variant
#define FX_RES_MAXI_SMALL 7           // ... its instance for small boxes (fewer registers)
#define FX_RES_MAXZ 10                // interior planes per thread column, faces-first column variant
#define FX_RES_SMEM_MAX (226 * 1024)  // dynamic shared memory per CTA (227 KB opt-in less static)
#define FX_RES_SPIN_LIMIT (1u << 24)  // polls of a neighbour's flag (well over a second with back-off)
#define FX_RES_MAX_CTAS 1024          // boxes per simulation and phase (flag slots)
#define FX_RES_FLAGS 16               // offset of the flag slots in FxSimDev::sync
#define FX_RES_SYNC_WORDS (FX_RES_FLAGS + 2 * FX_RES_MAX_CTAS)
// Words of FxSimDev::sync after the error word [2], set from the host (firex_set_wait_limit,
// firex_test_hold_face) and zero by default:
//   [3] polls of a neighbour's flag before a wait gives up (0: FX_RES_SPIN_LIMIT);
//   [4] box + 1 that stops publishing its faces from sweep [5] on (0: every box publishes) —
//       a flag that nothing sets (the flags only grow, so a single withheld sweep would only
//       delay the neighbours), so their bounded waits expire (test of the error path).
#define FX_SYNC_SPIN 3
#define FX_SYNC_HOLD_BOX 4
#define FX_SYNC_HOLD_SWEEP 5

// Shared-memory bytes of a box: pressure with halo rows + divergence.
__host__ __device__ inline long long fx_res_smem_bytes(int X, int by, int bz) {
    return ((long long)(by + 2) * (bz + 2) + (long long)by * bz) * X * 4;
}

FXD unsigned fx_ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Four consecutive pressure elements through L2 only (written by other SMs this launch).
template <typename PT>
FXD float4 fx_res_ld4_cg(const void* b, long long i);
template <>
FXD float4 fx_res_ld4_cg<float>(const void* b, long long i) {
    return __ldcg(reinterpret_cast<const float4*>(reinterpret_cast<const float*>(b) + i));
}
template <>
FXD float4 fx_res_ld4_cg<__half>(const void* b, long long i) {
    uint2 r = __ldcg(reinterpret_cast<const uint2*>(reinterpret_cast<const __half*>(b) + i));
    float2 a = __half22float2(*reinterpret_cast<__half2*>(&r.x));
    float2 c = __half22float2(*reinterpret_cast<__half2*>(&r.y));
    return make_float4(a.x, a.y, c.x, c.y);
}

FXD void fx_st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// The sync words of the simulation whose error word is `err`.
FXD const unsigned* fx_res_sync(const unsigned* err) { return err - 2; }

// Polls before a wait gives up.
FXD unsigned fx_res_spin_limit(const unsigned* err) {
    const unsigned v = fx_res_sync(err)[FX_SYNC_SPIN];
    return v ? v : FX_RES_SPIN_LIMIT;
}

// Variant 3 publishes per warp: each warp adds 1 to its box's flag (a release add) once its own
// face stores are done, so no CTA barrier precedes the publication; a box has published sweep s
// when its flag reaches FX_RES_WARPS * (s + 1) (the acquire load that sees that count sees
// every warp's stores: each add heads a release sequence).
#ifndef FX_RES_WARP_PUBLISH
#define FX_RES_WARP_PUBLISH 1
#endif
#define FX_RES_WARPS (FX_RES_THREADS / 32)
FXD void fx_red_release_add_u32(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
FXD void fx_res_publish_warp(unsigned* flags, int me, unsigned s, const unsigned* err) {
    const unsigned* sync = err - 2;
    if (sync[FX_SYNC_HOLD_BOX] == (unsigned)me + 1 && s >= sync[FX_SYNC_HOLD_SWEEP]) return;
    fx_red_release_add_u32(flags + me, 1u);
}

// Publishes box `me`'s faces of sweep s (flag = s + 1, release), unless the host holds them back.
FXD void fx_res_publish(unsigned* flags, int me, unsigned s, const unsigned* err) {
    const unsigned* sync = fx_res_sync(err);
    if (sync[FX_SYNC_HOLD_BOX] == (unsigned)me + 1 && s >= sync[FX_SYNC_HOLD_SWEEP]) return;
    fx_st_release_u32(flags + me, s + 1);
}

// Waits until each neighbour box has published sweep s (flag >= s + 1: acquire loads, one
// thread per neighbour, each wait bounded), then synchronises the CTA. False when a wait
// expired (the error word is then set).
FXD bool fx_res_wait(const unsigned* flags, const int nb[4], unsigned s, unsigned* err, int* flag) {
    if (threadIdx.x == 0) *flag = 1;
    __syncthreads();
    if (threadIdx.x < 4 && nb[threadIdx.x] >= 0) {
        const unsigned limit = fx_res_spin_limit(err);
        unsigned spins = 0;
        while (fx_ld_acquire_u32(flags + nb[threadIdx.x]) < s + 1) {
            if (++spins > limit) {
                atomicExch(err, 1u);
                *flag = 0;
                break;
            }
            if (spins > 64) __nanosleep(32);
        }
    }
    __syncthreads();
    return *flag != 0;
}

// Publishes this CTA's faces of sweep s (flag = s + 1, a release store after the CTA
// barrier, so every thread's face stores are visible first) and waits until each
// neighbour box has published sweep s (acquire loads, one thread per neighbour, each
// wait bounded). False when a wait expired (the error word is then set).
FXD bool fx_res_exchange(unsigned* flags, int me, const int nb[4], unsigned s, unsigned* err, int* flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        *flag = 1;
        fx_res_publish(flags, me, s, err);
    }
    __syncthreads();
    if (threadIdx.x < 4 && nb[threadIdx.x] >= 0) {
        const unsigned limit = fx_res_spin_limit(err);
        unsigned spins = 0;
        while (fx_ld_acquire_u32(flags + nb[threadIdx.x]) < s + 1) {
            if (++spins > limit) {
                atomicExch(err, 1u);
                *flag = 0;
                break;
            }
            if (spins > 64) __nanosleep(32);
        }
    }
    __syncthreads();
    return *flag != 0;
}

// Bounded wait until a neighbour's flag reaches `need` (acquire). False when it ran out.
FXD bool fx_res_wait_flag(const unsigned* flag, unsigned need, unsigned limit) {
    unsigned spins = 0;
    while (fx_ld_acquire_u32(flag) < need) {
        if (++spins > limit) return false;
        if (spins > 64) __nanosleep(32);
    }
    return true;
}

// Geometry of CTA b's box and its neighbours, and the box's first load.
struct FxResCtx {
    int X, Y, Z, n, y0, z0, ny, nz, gx, rowsP;
    long long XY;
    float *sp, *sd;  // pressure [(lz+1)*rowsP + ly+1][X] with halo rows; divergence [lz*by + ly][X]
    bool nbLoY, nbHiY, nbLoZ, nbHiZ;
    int nb[4];       // neighbour boxes within the group (-1: none)
    unsigned* flags;
    unsigned* err;
};

template <typename PT>
FXD FxResCtx fx_res_setup(const FxSimDev& S, const FxResBox& bx, int b, int phase, float* sm, bool load = true) {
    FxResCtx c;
    c.n = phase == 0 ? S.P : S.R;
    c.X = S.X;
    c.Y = S.Y;
    c.Z = S.Z;
    c.XY = (long long)c.X * c.Y;
    const int iy = b % bx.nby, iz = b / bx.nby;
    c.y0 = iy * bx.by;
    c.z0 = iz * bx.bz;
    c.ny = min(bx.by, c.Y - c.y0);
    c.nz = min(bx.bz, c.Z - c.z0);
    c.gx = c.X >> 2;
    c.rowsP = bx.by + 2;
    c.sp = sm;
    c.sd = sm + (long long)(bx.bz + 2) * c.rowsP * c.X;
    c.nbLoY = c.y0 > 0;
    c.nbHiY = c.y0 + c.ny < c.Y;
    c.nbLoZ = c.z0 > 0;
    c.nbHiZ = c.z0 + c.nz < c.Z;
    c.nb[0] = c.nbLoY ? b - 1 : -1;
    c.nb[1] = c.nbHiY ? b + 1 : -1;
    c.nb[2] = c.nbLoZ ? b - bx.nby : -1;
    c.nb[3] = c.nbHiZ ? b + bx.nby : -1;
    c.flags = S.sync + FX_RES_FLAGS + phase * FX_RES_MAX_CTAS;
    c.err = S.sync + 2;
    if (!load) return c;  // variant 4's copy warp loads the box (fx_res_boot)
    // the box with its halo rows (clamped rows outside the grid are never read) and its divergence
    const FxSolveBufs b0 = fx_solve_bufs(S, phase, 0);
    const int gx = c.gx, ny = c.ny, nz = c.nz, X = c.X;
    const int rows = (nz + 2) * (ny + 2);
    for (int i = threadIdx.x; i < rows * gx; i += blockDim.x) {
        const int row = i / gx, q = i - row * gx;
        const int lz = row / (ny + 2) - 1, ly = row % (ny + 2) - 1;
        const int cz = min(max(c.z0 + lz, 0), c.Z - 1), cy = min(max(c.y0 + ly, 0), c.Y - 1);
        float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (!b0.zeroIn) v = PStore<PT>::ld4(b0.pin, cz * c.XY + (long long)cy * X + 4 * q);
        *reinterpret_cast<float4*>(c.sp + ((lz + 1) * c.rowsP + ly + 1) * X + 4 * q) = v;
    }
    for (int i = threadIdx.x; i < nz * ny * gx; i += blockDim.x) {
        const int row = i / gx, q = i - row * gx;
        const int lz = row / ny, ly = row - lz * ny;
        *reinterpret_cast<float4*>(c.sd + (lz * bx.by + ly) * X + 4 * q) =
            __ldg(reinterpret_cast<const float4*>(S.div + (c.z0 + lz) * c.XY + (long long)(c.y0 + ly) * X + 4 * q));
    }
    return c;
}

// Halo rows of the next sweep from the neighbours' faces in `pout`, then a CTA barrier.
template <typename PT>
FXD void fx_res_halo(const FxResCtx& c, const void* pout) {
    const int gx = c.gx, ny = c.ny, nz = c.nz, X = c.X;
    const int hy = (c.nbLoY ? nz : 0) + (c.nbHiY ? nz : 0);
    const int hz = (c.nbLoZ ? ny : 0) + (c.nbHiZ ? ny : 0);
    for (int i = threadIdx.x; i < (hy + hz) * gx; i += blockDim.x) {
        const int row = i / gx, q = i - row * gx;
        int ly, lz;
        if (row < hy) {
            const bool lo = c.nbLoY && row < nz;
            lz = lo ? row : row - (c.nbLoY ? nz : 0);
            ly = lo ? -1 : ny;
        } else {
            const int r = row - hy;
            const bool lo = c.nbLoZ && r < ny;
            ly = lo ? r : r - (c.nbLoZ ? ny : 0);
            lz = lo ? -1 : nz;
        }
        const float4 v = fx_res_ld4_cg<PT>(pout, (c.z0 + lz) * c.XY + (long long)(c.y0 + ly) * X + 4 * q);
        *reinterpret_cast<float4*>(c.sp + ((lz + 1) * c.rowsP + ly + 1) * X + 4 * q) = v;
    }
    __syncthreads();
}

// Halo item i (see fx_res_halo): global index and shared offset of its 4-cell group.
FXD void fx_res_halo_item(const FxResCtx& c, int i, long long& g, int& so) {
    const int gx = c.gx, ny = c.ny, nz = c.nz, X = c.X;
    const int hy = (c.nbLoY ? nz : 0) + (c.nbHiY ? nz : 0);
    const int row = i / gx, q = i - row * gx;
    int ly, lz;
    if (row < hy) {
        const bool lo = c.nbLoY && row < nz;
        lz = lo ? row : row - (c.nbLoY ? nz : 0);
        ly = lo ? -1 : ny;
    } else {
        const int r = row - hy;
        const bool lo = c.nbLoZ && r < ny;
        ly = lo ? r : r - (c.nbLoZ ? ny : 0);
        lz = lo ? -1 : nz;
    }
    g = (c.z0 + lz) * c.XY + (long long)(c.y0 + ly) * X + 4 * q;
    so = ((lz + 1) * c.rowsP + ly + 1) * X + 4 * q;
}
FXD int fx_res_halo_total(const FxResCtx& c) {
    const int hy = (c.nbLoY ? c.nz : 0) + (c.nbHiY ? c.nz : 0);
    const int hz = (c.nbLoZ ? c.ny : 0) + (c.nbHiZ ? c.ny : 0);
    return (hy + hz) * c.gx;
}

// Column variant: thread t takes the box's (x group, row) column t and walks its z planes
// with the z neighbours in registers; the CTA publishes all faces after the whole sweep.
// For boxes with up to FX_RES_MAXG planes per thread column (the HD tier's 16 x 11 rows).
template <typename PT, bool ROUND>
FXD void fx_res_box_col(const FxSimDev& S, const FxResBox& bx, int b, int phase, float* sm) {
    __shared__ int s_flag;
    const FxResCtx cx = fx_res_setup<PT>(S, bx, b, phase, sm);
    const int n = cx.n, X = cx.X, Y = cx.Y, Z = cx.Z, y0 = cx.y0, z0 = cx.z0, ny = cx.ny, nz = cx.nz, gx = cx.gx;
    const int rowsP = cx.rowsP;
    const long long XY = cx.XY;
    float* sp = cx.sp;
    const float* sd = cx.sd;
    const bool nbLoY = cx.nbLoY, nbHiY = cx.nbHiY, nbLoZ = cx.nbLoZ, nbHiZ = cx.nbHiZ;
    // ---- this thread's z column: groups (q, ly, lz) for lz in [zs, zs + cnt). Columns
    // (q, ly) are spread over the threads, each split into P parts along z when there are
    // fewer columns than threads; the planner keeps cnt <= FX_RES_MAXG.
    const int C = gx * ny;
    const int P = max(1, (int)blockDim.x / C);
    const int zlen = (nz + P - 1) / P;
    const int t = threadIdx.x;
    const int col = t % C, part = t / C;
    const int q = col % gx, ly = col / gx, x0 = 4 * q;
    const int zs = part * zlen;
    const int cnt = (part < P) ? max(0, min(zlen, nz - zs)) : 0;
    const int y = y0 + ly;
    const bool top = y == Y - 1;  // the open top is the ambient-pressure boundary
    const int planeP = rowsP * X, planeD = bx.by * X;
    const int offC = ((zs + 1) * rowsP + ly + 1) * X + x0;  // smem offset of (x0, ly, zs)
    const int offD = (zs * bx.by + ly) * X + x0;
    const int offB = y > 0 ? -X : 0;
    const bool hasL = x0 > 0, hasR = x0 + 4 < X;
    const bool faceY = (ly == 0 && nbLoY) || (ly == ny - 1 && nbHiY);
    const long long gRow = (long long)(z0 + zs) * XY + (long long)y * X + x0;  // global index of (x0, y, z0+zs)
    const FxJacobiConst2 c2 = fx_jacobi_const2(FxJacobiConst{S.jc[0], S.jc[1], S.jc[2], S.jc[3]}, S.jcRcp, S.jcFastDiv != 0);
    __syncthreads();

    for (int s = 0; s < n; ++s) {
        float4 nv[FX_RES_MAXG];
        if (cnt > 0) {
            float4 pc = *reinterpret_cast<const float4*>(sp + offC);
            float4 pk = (z0 + zs > 0) ? *reinterpret_cast<const float4*>(sp + offC - planeP) : pc;
#pragma unroll
            for (int k = 0; k < FX_RES_MAXG; ++k) {
                if (k < cnt) {
                    const int off = offC + k * planeP;
                    const float4 pf = (z0 + zs + k < Z - 1) ? *reinterpret_cast<const float4*>(sp + off + planeP) : pc;
                    const float4 pb = *reinterpret_cast<const float4*>(sp + off + offB);
                    const float4 pt = *reinterpret_cast<const float4*>(sp + off + X);
                    const float pl = hasL ? sp[off - 1] : pc.x;
                    const float pr = hasR ? sp[off + 4] : pc.w;
                    const float4 d = *reinterpret_cast<const float4*>(sd + offD + k * planeD);
                    float4 o = fx_jacobi4<true>(c2, pl, pc, pr, pb, pt, pk, pf, d);
                    if (ROUND) o = make_float4(PStore<__half>::round(o.x), PStore<__half>::round(o.y),
                                               PStore<__half>::round(o.z), PStore<__half>::round(o.w));
                    nv[k] = top ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : o;
                    pk = pc;
                    pc = pf;
                }
            }
        }
        __syncthreads();  // every read of the old values is done
        const bool last = s == n - 1;
        const bool full = s >= n - 2;  // the last two sweeps fill both buffers of the pair
        void* pout = fx_solve_bufs(S, phase, s).pout;
#pragma unroll
        for (int k = 0; k < FX_RES_MAXG; ++k) {
            if (k < cnt) {
                *reinterpret_cast<float4*>(sp + offC + k * planeP) = nv[k];
                const int lz = zs + k;
                const bool face = faceY || (lz == 0 && nbLoZ) || (lz == nz - 1 && nbHiZ);
                if (full || face) PStore<PT>::st4(pout, gRow + (long long)k * XY, nv[k]);
            }
        }
        if (last) break;
        if (!fx_res_exchange(cx.flags, b, cx.nb, (unsigned)s, cx.err, &s_flag)) return;
        fx_res_halo<PT>(cx, pout);
    }
}

// Faces-first variant: the face groups are dealt out over all threads and computed
// first, stored and published before the interior is computed, so the flag travels while
// the CTA works. For boxes with at most FX_RES_MAXF face groups and FX_RES_MAXI interior
// groups per thread.
template <typename PT, bool ROUND, int MAXI>
FXD void fx_res_box_early(const FxSimDev& S, const FxResBox& bx, int b, int phase, float* sm) {
    __shared__ int s_flag;
    const FxResCtx cx = fx_res_setup<PT>(S, bx, b, phase, sm);
    const int n = cx.n, X = cx.X, Y = cx.Y, Z = cx.Z, y0 = cx.y0, z0 = cx.z0, ny = cx.ny, nz = cx.nz, gx = cx.gx;
    const int rowsP = cx.rowsP;
    const long long XY = cx.XY;
    float* sp = cx.sp;
    const float* sd = cx.sd;
    const bool nbLoY = cx.nbLoY, nbHiY = cx.nbHiY, nbLoZ = cx.nbLoZ, nbHiZ = cx.nbHiZ;
    // ---- this thread's groups of 4 x cells. The face groups (those a neighbour box reads:
    // y rows 0 / ny-1 and z planes 0 / nz-1 that have a neighbour) come first, then the
    // interior ones; each list is dealt out round-robin over the threads, so every thread
    // holds ceil(F/T) face slots then ceil(I/T) interior slots (the planner keeps their sum
    // within FX_RES_MAXF and MAXI). Packed as q | ly << 10 | lz << 21, -1 when empty.
    const int T = blockDim.x, t = threadIdx.x;
    const int fy0 = nbLoY ? 0 : -1, fy1 = (nbHiY && !(ny == 1 && nbLoY)) ? ny - 1 : -1;
    const int fz0 = nbLoZ ? 0 : -1, fz1 = (nbHiZ && !(nz == 1 && nbLoZ)) ? nz - 1 : -1;
    const int nyf = (fy0 >= 0) + (fy1 >= 0), nzf = (fz0 >= 0) + (fz1 >= 0);
    const int lyA = nbLoY ? 1 : 0, nyi = max(0, (nbHiY ? ny - 1 : ny) - lyA);  // rows off the y faces
    const int lzA = nbLoZ ? 1 : 0, nzi = max(0, (nbHiZ ? nz - 1 : nz) - lzA);  // planes off the z faces
    const int FY = nyf * nz * gx, F = FY + nzf * nyi * gx, I = nzi * nyi * gx;
    int pf[FX_RES_MAXF], pi[MAXI];  // this thread's face / interior groups
#pragma unroll
    for (int k = 0; k < FX_RES_MAXF; ++k) {
        const int i = t + k * T;
        int q = 0, ly = 0, lz = 0;
        if (i < FY) {
            q = i % gx;
            const int r = i / gx;
            lz = r % nz;
            ly = (r / nz == 0 && fy0 >= 0) ? fy0 : fy1;
        } else if (i < F) {
            const int j = i - FY;
            q = j % gx;
            const int r = j / gx;
            ly = lyA + r % nyi;
            lz = (r / nyi == 0 && fz0 >= 0) ? fz0 : fz1;
        }
        pf[k] = i < F ? (q | (ly << 10) | (lz << 21)) : -1;
    }
#pragma unroll
    for (int k = 0; k < MAXI; ++k) {
        const int j = t + k * T;
        int q = 0, ly = 0, lz = 0;
        if (j < I) {
            q = j % gx;
            const int r = j / gx;
            ly = lyA + r % nyi;
            lz = lzA + r / nyi;
        }
        pi[k] = j < I ? (q | (ly << 10) | (lz << 21)) : -1;
    }
    const FxJacobiConst2 c2 = fx_jacobi_const2(FxJacobiConst{S.jc[0], S.jc[1], S.jc[2], S.jc[3]}, S.jcRcp, S.jcFastDiv != 0);
    const int planeP = rowsP * X;
    // The packed coordinates pass through an empty asm on every use, so the compiler
    // recomputes the offsets each sweep instead of keeping one set per slot live across
    // the sweep loop (which spills).
    auto fresh = [](int g) {
        asm volatile("" : "+r"(g));
        return g;
    };
    // new value of group pk from the old values in shared memory
    auto update = [&](int g) {
        const int q = g & 0x3ff, ly = (g >> 10) & 0x7ff, lz = g >> 21;
        const int y = y0 + ly, z = z0 + lz, x0 = 4 * q;
        if (y == Y - 1) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // the open top is the ambient boundary
        const float* rowC = sp + ((lz + 1) * rowsP + ly + 1) * X;
        const float4 pc = *reinterpret_cast<const float4*>(rowC + x0);
        const float pl = x0 > 0 ? rowC[x0 - 1] : pc.x;
        const float pr = x0 + 4 < X ? rowC[x0 + 4] : pc.w;
        const float4 pb = *reinterpret_cast<const float4*>((y > 0 ? rowC - X : rowC) + x0);
        const float4 pt = *reinterpret_cast<const float4*>(rowC + X + x0);
        const float4 pkv = *reinterpret_cast<const float4*>((z > 0 ? rowC - planeP : rowC) + x0);
        const float4 pf = *reinterpret_cast<const float4*>((z < Z - 1 ? rowC + planeP : rowC) + x0);
        const float4 d = *reinterpret_cast<const float4*>(sd + (lz * bx.by + ly) * X + x0);
        float4 o = fx_jacobi4<true>(c2, pl, pc, pr, pb, pt, pkv, pf, d);
        if (ROUND) o = make_float4(PStore<__half>::round(o.x), PStore<__half>::round(o.y), PStore<__half>::round(o.z),
                                   PStore<__half>::round(o.w));
        return o;
    };
    auto gidx = [&](int g) {
        const int q = g & 0x3ff, ly = (g >> 10) & 0x7ff, lz = g >> 21;
        return (z0 + lz) * XY + (long long)(y0 + ly) * X + 4 * q;
    };
    auto sidx = [&](int g) {
        const int q = g & 0x3ff, ly = (g >> 10) & 0x7ff, lz = g >> 21;
        return ((lz + 1) * rowsP + ly + 1) * X + 4 * q;
    };
    // halo slot a face group is parked in: the one beyond its face (y rows first: a group on
    // a y face row belongs to the y list even when it also lies on a z face)
    auto parked = [&](int g) {
        const int q = g & 0x3ff;
        int ly = (g >> 10) & 0x7ff, lz = g >> 21;
        if (ly == fy0 || ly == fy1) ly = ly == fy0 ? -1 : ny;
        else lz = lz == fz0 ? -1 : nz;
        return ((lz + 1) * rowsP + ly + 1) * X + 4 * q;
    };
    __syncthreads();

    for (int s = 0; s < n; ++s) {
        const bool last = s == n - 1;
        const bool full = s >= n - 2;  // the last two sweeps fill both buffers of the pair
        void* pout = fx_solve_bufs(S, phase, s).pout;
        // faces first: computed, then parked in the halo slot next to them (no group reads a
        // halo slot once the face groups are done) and stored for the neighbours, and the
        // flag published before the interior is computed. Parking keeps the face values out
        // of registers while the interior ones are live.
        {
            float4 nf[FX_RES_MAXF];
#pragma unroll
            for (int k = 0; k < FX_RES_MAXF; ++k)
                if (pf[k] >= 0) nf[k] = update(fresh(pf[k]));
            __syncthreads();  // every read of a halo slot is done
#pragma unroll
            for (int k = 0; k < FX_RES_MAXF; ++k) {
                if (pf[k] >= 0) {
                    *reinterpret_cast<float4*>(sp + parked(fresh(pf[k]))) = nf[k];
                    if (!last) PStore<PT>::st4(pout, gidx(fresh(pf[k])), nf[k]);
                }
            }
        }
        if (!last) {
            __syncthreads();  // every face store of this CTA precedes the flag (release is cumulative)
            if (t == 0) fx_res_publish(cx.flags, b, (unsigned)s, cx.err);
        }
        float4 nv[MAXI];
#pragma unroll
        for (int k = 0; k < MAXI; ++k) {
            if (pi[k] >= 0) nv[k] = update(fresh(pi[k]));
            asm volatile("" ::: "memory");  // keep each group's loads with its update (register pressure)
        }
        __syncthreads();  // every read of the old values is done
#pragma unroll
        for (int k = 0; k < MAXI; ++k) {
            if (pi[k] >= 0) {
                *reinterpret_cast<float4*>(sp + sidx(fresh(pi[k]))) = nv[k];
                if (full) PStore<PT>::st4(pout, gidx(fresh(pi[k])), nv[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < FX_RES_MAXF; ++k) {
            if (pf[k] >= 0) {  // back from the slot this thread parked it in
                const float4 v = *reinterpret_cast<const float4*>(sp + parked(fresh(pf[k])));
                *reinterpret_cast<float4*>(sp + sidx(fresh(pf[k]))) = v;
                if (last) PStore<PT>::st4(pout, gidx(fresh(pf[k])), v);
            }
        }
        if (last) break;
        if (!fx_res_wait(cx.flags, cx.nb, (unsigned)s, cx.err, &s_flag)) return;
        fx_res_halo<PT>(cx, pout);
    }
}

// Variant 4's copy warp (the CTA's last warp; the other T threads run variant 3's sweep):
// for every sweep but the last, once the compute warps have read the halo rows of the sweep
// (they arrive on `faces` after their face groups, the only groups that read them), lanes
// 0-3 wait for the four neighbours' faces of the sweep (acquire loads of the flags, each
// bounded), and the lanes issue one bulk copy each of the halo rows and planes from the
// sweep's output buffer into the halo slots, completing on `halo`; the compute threads wait
// for that phase before the next sweep. The copies thus run while the interior is computed.
// Not inlined: its registers then stay out of the compute threads' allocation (inlined, the
// sweep spills).
struct FxResCopyBars {
    unsigned long long faces;  // the compute warps read the sweep's halo (count T / 32)
    unsigned long long halo;   // the next sweep's halo rows landed (count 1 + transaction bytes)
    unsigned long long boot;   // the box's first load landed (count 1 + transaction bytes)
};

// Variant 4's compute threads before the first sweep: clear the box when the phase starts from
// zero, then wait for the copy warp's first load (false when the wait ran out; the error word is
// then set). Not inlined, as fx_res_boot.
static __device__ __noinline__ bool fx_res_boot_wait(const FxSimDev& S, const FxResCtx& cx, int phase, int T,
                                                     unsigned long long* bar) {
    if (fx_solve_bufs(S, phase, 0).zeroIn) {
        const int n4 = (cx.nz + 2) * cx.rowsP * cx.gx;
        for (int i = threadIdx.x; i < n4; i += T) reinterpret_cast<float4*>(cx.sp)[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else if (cx.y0 + cx.ny == cx.Y) {
        // the row above the grid: the top row's update is 0 whatever it reads there, but its
        // numerators should not meet stale bits (NaN would send them to the slow division)
        for (int i = threadIdx.x; i < (cx.nz + 2) * cx.gx; i += T) {
            const int lz = i / cx.gx, q = i - lz * cx.gx;
            reinterpret_cast<float4*>(cx.sp + (lz * cx.rowsP + cx.ny + 1) * cx.X)[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
    const bool ok = fx_mbar_wait_bounded(bar, 0u, fx_res_spin_limit(cx.err));
    if (!ok) atomicExch(cx.err, 1u);
    return ok;
}

// Variant 4's first load of the box, by the copy warp: per plane of the box and its halo that
// lies in the grid, one bulk copy of its rows y0 - 1 .. y0 + ny that lie in the grid (they are
// contiguous in the field and in the box), and per plane one copy of the divergence rows,
// completing on `boot`. Rows and planes outside the grid are never read by the sweep (the walls
// take the cell itself, the top row is 0), so they are not loaded. A phase that starts from
// zero loads no pressure (the compute threads clear the box). The warp waits for its copies.
static __device__ __noinline__ void fx_res_boot(const FxSimDev& S, const FxResBox& bx, const FxResCtx& cx, int phase,
                                                unsigned long long* bar) {
    const int lane = threadIdx.x & 31;
    const FxSolveBufs b0 = fx_solve_bufs(S, phase, 0);
    const float* pin = reinterpret_cast<const float*>(b0.pin);
    const int X = cx.X, Y = cx.Y, Z = cx.Z, y0 = cx.y0, z0 = cx.z0, ny = cx.ny, nz = cx.nz, rowsP = cx.rowsP;
    const long long XY = cx.XY;
    const int ylo = max(y0 - 1, 0), yhi = min(y0 + ny + 1, Y);
    const int zlo = max(z0 - 1, 0), zhi = min(z0 + nz + 1, Z);
    const unsigned pBytes = (unsigned)(yhi - ylo) * (unsigned)X * 4u, dBytes = (unsigned)ny * (unsigned)X * 4u;
    const int np = b0.zeroIn ? 0 : zhi - zlo;
    if (lane == 0) fx_mbar_expect_tx(bar, (unsigned)np * pBytes + (unsigned)nz * dBytes);
    __syncwarp();
    for (int i = lane; i < np + nz; i += 32) {
        if (i < np) {
            const int z = zlo + i, lz = z - z0;
            fx_bulk_g2s(cx.sp + ((lz + 1) * rowsP + (ylo - y0 + 1)) * X, pin + (long long)z * XY + (long long)ylo * X, pBytes,
                        bar);
        } else {
            const int lz = i - np;
            fx_bulk_g2s(cx.sd + lz * bx.by * X, S.div + (long long)(z0 + lz) * XY + (long long)y0 * X, dBytes, bar);
        }
    }
    fx_mbar_wait_bounded(bar, 0u, fx_res_spin_limit(cx.err));
}
static __device__ __noinline__ void fx_res_copier(const FxSimDev& S, const FxResCtx& cx, int phase, int T, FxResCopyBars& bars,
                       volatile int* abort, bool epi) {
    const int n = cx.n, X = cx.X, y0 = cx.y0, z0 = cx.z0, ny = cx.ny, nz = cx.nz, rowsP = cx.rowsP;
    const long long XY = cx.XY;
    const int lane = threadIdx.x & 31;
    const unsigned limit = fx_res_spin_limit(cx.err), nw = (unsigned)T / 32u;
    const unsigned rowBytes = (unsigned)X * 4u, planeBytes = (unsigned)ny * rowBytes;
    const int nbMine = lane == 0 ? cx.nb[0] : lane == 1 ? cx.nb[1] : lane == 2 ? cx.nb[2] : lane == 3 ? cx.nb[3] : -1;
    const unsigned bytes = (unsigned)nz * rowBytes * ((cx.nbLoY ? 1u : 0u) + (cx.nbHiY ? 1u : 0u)) +
                           planeBytes * ((cx.nbLoZ ? 1u : 0u) + (cx.nbHiZ ? 1u : 0u));
    int armed = 0;  // sweeps whose halo was requested
    bool ok = true;
    // with the projection epilogue, the last sweep's faces are fetched too (its halo rows)
    for (int s = 0; s + (epi ? 0 : 1) < n; ++s) {
        const float* pout = reinterpret_cast<const float*>(fx_solve_bufs(S, phase, s).pout);
        bool mine = fx_mbar_wait_bounded(&bars.faces, (unsigned)s & 1u, limit);
        if (mine && nbMine >= 0) mine = fx_res_wait_flag(cx.flags + nbMine, nw * ((unsigned)s + 1u), limit);
        if (!__all_sync(0xffffffffu, mine)) {
            ok = false;
            break;
        }
        // the neighbours' face stores, seen through lanes 0-3's acquire loads and the warp
        // barrier, come before the copies; the compute warps' reads of the slots are ordered
        // by the faces mbarrier
        fx_fence_proxy_async_global();
        if (lane == 0) fx_mbar_expect_tx(&bars.halo, bytes);
        __syncwarp();
        armed = s + 1;
        for (int i = lane; i < 2 * nz + 2; i += 32) {
            if (i < nz) {
                if (cx.nbLoY)
                    fx_bulk_g2s(cx.sp + (i + 1) * rowsP * X, pout + (long long)(z0 + i) * XY + (long long)(y0 - 1) * X,
                                rowBytes, &bars.halo);
            } else if (i < 2 * nz) {
                const int lz = i - nz;
                if (cx.nbHiY)
                    fx_bulk_g2s(cx.sp + ((lz + 1) * rowsP + ny + 1) * X,
                                pout + (long long)(z0 + lz) * XY + (long long)(y0 + ny) * X, rowBytes, &bars.halo);
            } else if (i == 2 * nz) {
                if (cx.nbLoZ)
                    fx_bulk_g2s(cx.sp + X, pout + (long long)(z0 - 1) * XY + (long long)y0 * X, planeBytes, &bars.halo);
            } else if (cx.nbHiZ) {
                fx_bulk_g2s(cx.sp + ((nz + 1) * rowsP + 1) * X, pout + (long long)(z0 + nz) * XY + (long long)y0 * X,
                            planeBytes, &bars.halo);
            }
        }
    }
    if (!ok && lane == 0) {
        atomicExch(cx.err, 1u);
        *abort = 1;
    }
    // every copy this warp issued lands before the CTA can end
    if (armed > 0) fx_mbar_wait_bounded(&bars.halo, (unsigned)(armed - 1) & 1u, limit);
}

// Variant 4's projection epilogue of the residual phase (projectVelocity with the correction,
// fxk_project phase 1, with its operations): after the last sweep the box holds the final
// correction and its halo rows the neighbours' final faces, so each group of 4 cells of a box
// row reads its flow from global memory and writes the projected flow, every pressure from
// shared memory. The top row takes the projection of the row below (the planner gives the top
// box at least two rows, so that row and its plane in front are in the box or its halo).
// Not inlined: it keeps the sweep's register allocation.
static __device__ __noinline__ void fx_res_project_epi(const FxSimDev& S, const FxResCtx& cx, int T) {
    const float4* __restrict__ flowIn = reinterpret_cast<const float4*>(S.flow[S.fi]);
    float4* __restrict__ flowOut = reinterpret_cast<float4*>(S.flow[S.fi ^ 1]);
    const float3 m = fx_metric(S.prm.u);
    const int X = cx.X, Y = cx.Y, Z = cx.Z, gx = cx.gx, ny = cx.ny, rowsP = cx.rowsP;
    const long long XY = cx.XY;
    const int planeP = rowsP * X;
    const int total = ny * cx.nz * gx;
    for (int i = threadIdx.x; i < total; i += T) {
        const int q = i % gx, r = i / gx, ly = r % ny, lz = r / ny;
        const int y = cx.y0 + ly, z = cx.z0 + lz, x0 = 4 * q;
        const bool topRow = y == Y - 1;
        const long long c = (long long)z * XY + (long long)y * X + x0;
        const long long cs = topRow ? c - X : c;  // top row: the projected row below
        const float* rowS = cx.sp + ((lz + 1) * rowsP + (topRow ? ly - 1 : ly) + 1) * X;
        const float4 pc4 = *reinterpret_cast<const float4*>(rowS + x0);
        const float p4 = x0 + 4 < X ? rowS[x0 + 4] : 0.0f;
        const float4 pt4 = *reinterpret_cast<const float4*>(rowS + X + x0);
        const float4 pf4 = z < Z - 1 ? *reinterpret_cast<const float4*>(rowS + planeP + x0) : pc4;
        float4 f[4], sv[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) f[j] = __ldg(flowIn + c + j);
#pragma unroll
        for (int j = 0; j < 4; ++j) sv[j] = topRow ? __ldg(flowIn + cs + j) : f[j];
        const float pcs[5] = {pc4.x, pc4.y, pc4.z, pc4.w, p4};
        const float pts[4] = {pt4.x, pt4.y, pt4.z, pt4.w}, pfs[4] = {pf4.x, pf4.y, pf4.z, pf4.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int x = x0 + j;
            const float pc = pcs[j];
            const float px = x + 1 < X ? pcs[j + 1] : pc;
            const float gxv = (px - pc) * m.x;
            const float gyv = (pts[j] - pc) * m.y;
            const float gzv = (pfs[j] - pc) * m.z;
            float4 o = make_float4(sv[j].x - gxv, sv[j].y - gyv, sv[j].z - gzv, f[j].w);
            if (x == 0 || x == X - 1) o.x = 0.0f;
            if (z == 0 || z == Z - 1) o.z = 0.0f;
            if (y == 0) o.y = 0.0f;
            if (y == Y - 1) o.y = fx_max(0.0f, o.y);
            flowOut[c + j] = o;
        }
    }
}

// Faces-first column variant: the face groups are dealt out over all threads as in the
// faces-first variant and kept in registers (no parking); the interior is walked in z
// columns, thread t taking interior column (x group, row) t with its z neighbours in
// registers, its x neighbours from the adjacent lanes (warp shuffles) where those hold
// the same row and plane.
// Two CTA barriers per sweep: old values read and neighbour flags seen (the waiting threads
// spin before it), new values and halo rows written; each warp publishes its own face stores
// with a release add (FX_RES_WARP_PUBLISH; otherwise a third barrier orders the CTA's face
// stores before one release store). Each thread's first halo load is issued before it writes its new values back,
// so that L2 round trip overlaps the write-back (0.8 % faster at HD). For boxes whose interior columns fit the threads (planner: at most
// FX_RES_MAXZ planes per column part).
// COPY (variant 4, FP32 pressure): the last warp is a copy warp (fx_res_copier) that waits for
// the neighbours and brings the halo rows in with bulk copies while the interior is computed;
// the other FX_RES_COPY_TC threads run the sweep, synchronise on a named barrier, publish per
// warp, and wait for the copies instead of waiting for flags and loading the halo themselves.
template <typename PT, bool ROUND, bool COPY, bool EPI = false>
FXD void fx_res_box_v3(const FxSimDev& S, const FxResBox& bx, int b, int phase, float* sm) {
    constexpr bool epi = EPI;
    __shared__ int s_flag;
    __shared__ FxResCopyBars cbars;
    __shared__ int s_abort;
    const FxResCtx cx = fx_res_setup<PT>(S, bx, b, phase, sm, !COPY);
    const int n = cx.n, X = cx.X, Y = cx.Y, Z = cx.Z, y0 = cx.y0, z0 = cx.z0, ny = cx.ny, nz = cx.nz, gx = cx.gx;
    const int rowsP = cx.rowsP;
    const long long XY = cx.XY;
    const bool nbLoY = cx.nbLoY, nbHiY = cx.nbHiY, nbLoZ = cx.nbLoZ, nbHiZ = cx.nbHiZ;
    const int T = (int)blockDim.x - (COPY ? 32 : 0), t = threadIdx.x, lane = t & 31;
    float* sp = cx.sp;
    const float* sd = cx.sd;
    const int planeP = rowsP * X, planeD = bx.by * X;
    // ---- face groups, as in fx_res_box_early
    const int fy0 = nbLoY ? 0 : -1, fy1 = (nbHiY && !(ny == 1 && nbLoY)) ? ny - 1 : -1;
    const int fz0 = nbLoZ ? 0 : -1, fz1 = (nbHiZ && !(nz == 1 && nbLoZ)) ? nz - 1 : -1;
    const int nyf = (fy0 >= 0) + (fy1 >= 0), nzf = (fz0 >= 0) + (fz1 >= 0);
    const int lyA = nbLoY ? 1 : 0, nyi = max(0, (nbHiY ? ny - 1 : ny) - lyA);
    const int lzA = nbLoZ ? 1 : 0, nzi = max(0, (nbHiZ ? nz - 1 : nz) - lzA);
    const int FY = nyf * nz * gx, F = FY + nzf * nyi * gx;
    int pf[FX_RES_MAXF];
#pragma unroll
    for (int k = 0; k < FX_RES_MAXF; ++k) {
        const int i = t + k * T;
        int q = 0, ly = 0, lz = 0;
        if (i < FY) {
            q = i % gx;
            const int r = i / gx;
            lz = r % nz;
            ly = (r / nz == 0 && fy0 >= 0) ? fy0 : fy1;
        } else if (i < F) {
            const int j = i - FY;
            q = j % gx;
            const int r = j / gx;
            ly = lyA + r % nyi;
            lz = (r / nyi == 0 && fz0 >= 0) ? fz0 : fz1;
        }
        pf[k] = i < F ? (q | (ly << 10) | (lz << 21)) : -1;
    }
    // ---- this thread's interior column: (q, ly) = column t % C, z part t / C
    const int C = nyi * gx;
    const int P = C > 0 ? max(1, T / C) : 1;
    const int zlen = (nzi + P - 1) / P;
    const int col = C > 0 ? t % C : 0, part = C > 0 ? t / C : P;
    const int q = col % gx, ly = lyA + col / gx, x0 = 4 * q;
    const int zs = lzA + part * zlen;
    const int cnt = part < P ? max(0, min(zlen, lzA + nzi - zs)) : 0;
    const int y = y0 + ly;
    const bool top = y == Y - 1;  // the open top is the ambient-pressure boundary
    const int offC = ((zs + 1) * rowsP + ly + 1) * X + x0;  // (x0, ly, zs)
    const int offD = (zs * bx.by + ly) * X + x0;
    const int offB = y > 0 ? -X : 0;
    const bool hasL = x0 > 0, hasR = x0 + 4 < X;
    // x neighbours from the adjacent lane when it holds the adjacent group of the same
    // row and z part (it then walks the same planes); else from shared memory
    const bool shflL = lane > 0 && q > 0 && col > 0 && part < P;
    const bool shflR = lane < 31 && q < gx - 1 && col < C - 1 && t + 1 < T && part < P;
    const long long gRow = (long long)(z0 + zs) * XY + (long long)y * X + x0;
    const FxJacobiConst2 c2 = fx_jacobi_const2(FxJacobiConst{S.jc[0], S.jc[1], S.jc[2], S.jc[3]}, S.jcRcp, S.jcFastDiv != 0);
    // new value of face group g from the old values in shared memory
    auto update = [&](int g) {
        const int fq = g & 0x3ff, fly = (g >> 10) & 0x7ff, flz = g >> 21;
        const int fyy = y0 + fly, fz = z0 + flz, fx0 = 4 * fq;
        if (fyy == Y - 1) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const float* rowC = sp + ((flz + 1) * rowsP + fly + 1) * X;
        const float4 pc = *reinterpret_cast<const float4*>(rowC + fx0);
        const float pl = fx0 > 0 ? rowC[fx0 - 1] : pc.x;
        const float pr = fx0 + 4 < X ? rowC[fx0 + 4] : pc.w;
        const float4 pb = *reinterpret_cast<const float4*>((fyy > 0 ? rowC - X : rowC) + fx0);
        const float4 pt = *reinterpret_cast<const float4*>(rowC + X + fx0);
        const float4 pkv = *reinterpret_cast<const float4*>((fz > 0 ? rowC - planeP : rowC) + fx0);
        const float4 pfv = *reinterpret_cast<const float4*>((fz < Z - 1 ? rowC + planeP : rowC) + fx0);
        const float4 d = *reinterpret_cast<const float4*>(sd + (flz * bx.by + fly) * X + fx0);
        float4 o = fx_jacobi4<true, COPY>(c2, pl, pc, pr, pb, pt, pkv, pfv, d);
        if (ROUND) o = make_float4(PStore<__half>::round(o.x), PStore<__half>::round(o.y), PStore<__half>::round(o.z),
                                   PStore<__half>::round(o.w));
        return o;
    };
    auto gidx = [&](int g) {
        const int fq = g & 0x3ff, fly = (g >> 10) & 0x7ff, flz = g >> 21;
        return (z0 + flz) * XY + (long long)(y0 + fly) * X + 4 * fq;
    };
    auto sidx = [&](int g) {
        const int fq = g & 0x3ff, fly = (g >> 10) & 0x7ff, flz = g >> 21;
        return ((flz + 1) * rowsP + fly + 1) * X + 4 * fq;
    };
    // With COPY the face slots pass through an empty asm on every use, so the compiler
    // recomputes their offsets each sweep instead of keeping them live across the sweep loop
    // (which spills); without it the plain values compile without spills.
    auto fresh = [](int g) {
        if (COPY) asm volatile("" : "+r"(g));
        return g;
    };
    if (t == 0) {
        s_flag = 1;
        if (COPY) {
            fx_mbar_init(&cbars.faces, (unsigned)T / 32u);
            fx_mbar_init(&cbars.halo, 1);
            fx_mbar_init(&cbars.boot, 1);
            s_abort = 0;
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
    }
    __syncthreads();
    if (COPY && t >= T) {
        fx_res_boot(S, bx, cx, phase, &cbars.boot);
        fx_res_copier(S, cx, phase, T, cbars, &s_abort, epi);
        return;
    }
    const unsigned limit = fx_res_spin_limit(cx.err);
    if (COPY && fx_bar_or(1, T, !fx_res_boot_wait(S, cx, phase, T, &cbars.boot))) return;

    for (int s = 0; s < n; ++s) {
        const bool last = s == n - 1;
        const bool full = s >= n - 2;  // the last two sweeps fill both buffers of the pair
        void* pout = fx_solve_bufs(S, phase, s).pout;
        float4 nf[FX_RES_MAXF];
#pragma unroll
        for (int k = 0; k < FX_RES_MAXF; ++k) {
            if (pf[k] >= 0) {
                const int g = fresh(pf[k]);
                nf[k] = update(g);
                if (!last || epi) PStore<PT>::st4(pout, gidx(g), nf[k]);
            }
        }
        if (!last || epi) {
            if (COPY) {
                __syncwarp();  // this warp's face stores and halo reads precede its add and arrival
                if (lane == 0) {
                    fx_res_publish_warp(cx.flags, b, (unsigned)s, cx.err);
                    fx_mbar_arrive(&cbars.faces);
                }
            } else if (FX_RES_WARP_PUBLISH) {
                __syncwarp();  // this warp's face stores precede its add (release is cumulative)
                if ((t & 31) == 0) fx_res_publish_warp(cx.flags, b, (unsigned)s, cx.err);
            } else {
                __syncthreads();  // every face store of this CTA precedes the flag
                if (t == 0) fx_res_publish(cx.flags, b, (unsigned)s, cx.err);
            }
        }
        float4 nv[FX_RES_MAXZ];
        {
            float4 pc = make_float4(0.0f, 0.0f, 0.0f, 0.0f), pk = pc;  // threads without a column load nothing
            if (cnt > 0) {
                pc = *reinterpret_cast<const float4*>(sp + offC);
                pk = (z0 + zs > 0) ? *reinterpret_cast<const float4*>(sp + offC - planeP) : pc;
            }
#pragma unroll
            for (int k = 0; k < FX_RES_MAXZ; ++k) {
                const bool v = k < cnt;
                const int off = offC + k * planeP;
                float4 pfv = pc;
                if (v && z0 + zs + k < Z - 1) pfv = *reinterpret_cast<const float4*>(sp + off + planeP);
                // every lane takes part in the shuffles; a value is used only from a lane of
                // the same row and part, which walks the same plane k
                const float fromL = __shfl_up_sync(0xffffffffu, pc.w, 1);
                const float fromR = __shfl_down_sync(0xffffffffu, pc.x, 1);
                if (v) {
                    const float4 pb = *reinterpret_cast<const float4*>(sp + off + offB);
                    const float4 pt = *reinterpret_cast<const float4*>(sp + off + X);
                    const float pl = shflL ? fromL : (hasL ? sp[off - 1] : pc.x);
                    const float pr = shflR ? fromR : (hasR ? sp[off + 4] : pc.w);
                    const float4 d = *reinterpret_cast<const float4*>(sd + offD + k * planeD);
                    float4 o = fx_jacobi4<true, COPY>(c2, pl, pc, pr, pb, pt, pk, pfv, d);
                    if (ROUND) o = make_float4(PStore<__half>::round(o.x), PStore<__half>::round(o.y),
                                               PStore<__half>::round(o.z), PStore<__half>::round(o.w));
                    nv[k] = top ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : o;
                }
                pk = pc;
                pc = pfv;
            }
        }
        // the neighbours' faces of this sweep: the waiting threads spin before the barrier
        // that also ends every read of the old values
        if (!COPY && !last && t < 4 && cx.nb[t] >= 0) {
            const unsigned limit = fx_res_spin_limit(cx.err);
            unsigned spins = 0;
            const unsigned need = FX_RES_WARP_PUBLISH ? FX_RES_WARPS * ((unsigned)s + 1) : (unsigned)s + 1;
            while (fx_ld_acquire_u32(cx.flags + cx.nb[t]) < need) {
                if (++spins > limit) {
                    atomicExch(cx.err, 1u);
                    s_flag = 0;
                    break;
                }
                if (spins > 64) __nanosleep(32);
            }
        }
        if (COPY) {
            if (fx_bar_or(1, T, *reinterpret_cast<volatile int*>(&s_abort) != 0)) return;
        } else {
            __syncthreads();
            if (!s_flag) return;  // a wait expired (every thread sees it after the barrier)
        }
        // the first halo item's load goes out before the write-back
        const int hTotal = (last || COPY) ? 0 : fx_res_halo_total(cx);
        float4 h0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        int h0so = -1;
        if (t < hTotal) {
            long long hg;
            fx_res_halo_item(cx, t, hg, h0so);
            h0 = fx_res_ld4_cg<PT>(pout, hg);
        }
        {
#pragma unroll
            for (int k = 0; k < FX_RES_MAXZ; ++k) {
                if (k < cnt) {
                    *reinterpret_cast<float4*>(sp + offC + k * planeP) = nv[k];
                    if (full) PStore<PT>::st4(pout, gRow + (long long)k * XY, nv[k]);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < FX_RES_MAXF; ++k) {
            if (pf[k] >= 0) {
                const int g = fresh(pf[k]);
                *reinterpret_cast<float4*>(sp + sidx(g)) = nf[k];
                if (last && !epi) PStore<PT>::st4(pout, gidx(g), nf[k]);
            }
        }
        if (last && !epi) break;
        if (COPY) {  // the copy warp's halo rows of this sweep
            const bool bad = !fx_mbar_wait_bounded(&cbars.halo, (unsigned)s & 1u, limit);
            if (bad) atomicExch(cx.err, 1u);
            if (fx_bar_or(1, T, bad || *reinterpret_cast<volatile int*>(&s_abort) != 0)) return;
            if (last) {  // epi: the final box and halo in place
                fx_res_project_epi(S, cx, T);
                break;
            }
        } else {
            if (h0so >= 0) *reinterpret_cast<float4*>(sp + h0so) = h0;
            for (int i = t + T; i < hTotal; i += T) {
                long long hg;
                int so;
                fx_res_halo_item(cx, i, hg, so);
                *reinterpret_cast<float4*>(sp + so) = fx_res_ld4_cg<PT>(pout, hg);
            }
            __syncthreads();  // halo rows in place before the next sweep
        }
    }
}
