// fx_jacobi_res.cuh — every sweep of one Jacobi phase (solvePressureGlobal,
// shaders.ts:375-403) in ONE cooperative launch, with the pressure resident on chip.
//
// Each simulation of the batch gets a group of CTAs (one per SM); CTA b of the group owns
// a box of by x bz rows (y, z) of full x rows and keeps the box's pressure, with a
// one-row halo on each side in y and z, and its divergence in shared memory for the
// whole phase. A sweep reads only shared memory: each thread computes its groups of 4
// consecutive x cells into registers, the CTA synchronises, then writes the new values
// back. Only box faces leave the SM: after every sweep but the last, the cells a
// neighbour box needs are stored to the sweep's output buffer, the CTA publishes a
// per-box flag (release store) and waits for the flags of its up to four neighbours
// (acquire loads, bounded waits), then loads its halo rows from that buffer through L2
// (ld.global.cg: L1 may hold stale lines). Only neighbours synchronise, so there is no
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
// arrives; the waits are still bounded (FX_RES_SPIN_LIMIT polls): on expiry the CTA
// sets the simulation's error word and returns, and the host reports a timeout.
#pragma once

#include "fx_step_math.cuh"
#include "fx_storage.cuh"

#define FX_RES_THREADS 512
#define FX_RES_MAXG 12                // groups of 4 cells per thread
#define FX_RES_SMEM_MAX (226 * 1024)  // dynamic shared memory per CTA (227 KB opt-in less static)
#define FX_RES_SPIN_LIMIT (1u << 24)  // polls of a neighbour's flag (well over a second with back-off)
#define FX_RES_MAX_CTAS 1024          // boxes per simulation and phase (flag slots)
#define FX_RES_FLAGS 16               // offset of the flag slots in FxSimDev::sync
#define FX_RES_SYNC_WORDS (FX_RES_FLAGS + 2 * FX_RES_MAX_CTAS)

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

// Publishes this CTA's faces of sweep s (flag = s + 1, a release store after the CTA
// barrier, so every thread's face stores are visible first) and waits until each
// neighbour box has published sweep s (acquire loads, one thread per neighbour, each
// wait bounded). False when a wait expired (the error word is then set).
FXD bool fx_res_exchange(unsigned* flags, int me, const int nb[4], unsigned s, unsigned* err, int* flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        *flag = 1;
        fx_st_release_u32(flags + me, s + 1);
    }
    __syncthreads();
    if (threadIdx.x < 4 && nb[threadIdx.x] >= 0) {
        unsigned spins = 0;
        while (fx_ld_acquire_u32(flags + nb[threadIdx.x]) < s + 1) {
            if (++spins > FX_RES_SPIN_LIMIT) {
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

// One CTA's share of a resident phase. PT: pressure storage; ROUND: round every sweep's
// output to FP16 (pressure stored in FP16).
template <typename PT, bool ROUND>
FXD void fx_res_box(const FxSimDev& S, const FxResBox& bx, int b, int phase, float* sm) {
    __shared__ int s_flag;
    const int n = phase == 0 ? S.P : S.R;
    const int X = S.X, Y = S.Y, Z = S.Z;
    const long long XY = (long long)X * Y;
    const int iy = b % bx.nby, iz = b / bx.nby;
    const int y0 = iy * bx.by, z0 = iz * bx.bz;
    const int ny = min(bx.by, Y - y0), nz = min(bx.bz, Z - z0);
    const int gx = X >> 2;
    const int rowsP = bx.by + 2;
    float* sp = sm;                                            // [(lz+1)*rowsP + ly+1][X]
    float* sd = sm + (long long)(bx.bz + 2) * rowsP * X;       // [lz*by + ly][X]
    const bool nbLoY = y0 > 0, nbHiY = y0 + ny < Y, nbLoZ = z0 > 0, nbHiZ = z0 + nz < Z;
    unsigned* flags = S.sync + FX_RES_FLAGS + phase * FX_RES_MAX_CTAS;
    unsigned* err = S.sync + 2;
    // neighbour boxes within the group (-1: none)
    const int nb[4] = {nbLoY ? b - 1 : -1, nbHiY ? b + 1 : -1, nbLoZ ? b - bx.nby : -1, nbHiZ ? b + bx.nby : -1};

    const FxSolveBufs b0 = fx_solve_bufs(S, phase, 0);
    // ---- load the box with its halo rows (clamped rows outside the grid are never read)
    {
        const int rows = (nz + 2) * (ny + 2);
        for (int i = threadIdx.x; i < rows * gx; i += blockDim.x) {
            const int row = i / gx, q = i - row * gx;
            const int lz = row / (ny + 2) - 1, ly = row % (ny + 2) - 1;
            const int cz = min(max(z0 + lz, 0), Z - 1), cy = min(max(y0 + ly, 0), Y - 1);
            float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (!b0.zeroIn) v = PStore<PT>::ld4(b0.pin, cz * XY + (long long)cy * X + 4 * q);
            *reinterpret_cast<float4*>(sp + ((lz + 1) * rowsP + ly + 1) * X + 4 * q) = v;
        }
        for (int i = threadIdx.x; i < nz * ny * gx; i += blockDim.x) {
            const int row = i / gx, q = i - row * gx;
            const int lz = row / ny, ly = row - lz * ny;
            *reinterpret_cast<float4*>(sd + (lz * bx.by + ly) * X + 4 * q) =
                __ldg(reinterpret_cast<const float4*>(S.div + (z0 + lz) * XY + (long long)(y0 + ly) * X + 4 * q));
        }
    }
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
                    float4 o = fx_jacobi4(c2, pl, pc, pr, pb, pt, pk, pf, d);
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
        if (!fx_res_exchange(flags, b, nb, (unsigned)s, err, &s_flag)) return;
        // ---- halo rows of the next sweep from the neighbours' faces
        const int hy = (nbLoY ? nz : 0) + (nbHiY ? nz : 0);
        const int hz = (nbLoZ ? ny : 0) + (nbHiZ ? ny : 0);
        for (int i = threadIdx.x; i < (hy + hz) * gx; i += blockDim.x) {
            const int row = i / gx, q = i - row * gx;
            int ly, lz;
            if (row < hy) {
                const bool lo = nbLoY && row < nz;
                lz = lo ? row : row - (nbLoY ? nz : 0);
                ly = lo ? -1 : ny;
            } else {
                const int r = row - hy;
                const bool lo = nbLoZ && r < ny;
                ly = lo ? r : r - (nbLoZ ? ny : 0);
                lz = lo ? -1 : nz;
            }
            const float4 v = fx_res_ld4_cg<PT>(pout, (z0 + lz) * XY + (long long)(y0 + ly) * X + 4 * q);
            *reinterpret_cast<float4*>(sp + ((lz + 1) * rowsP + ly + 1) * X + 4 * q) = v;
        }
        __syncthreads();
    }
}
