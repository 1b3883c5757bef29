// fx_jacobi_tb.cuh — temporally blocked Jacobi: K sweeps of solvePressureGlobal
// (shaders.ts:375-403) per launch, each sweep's update computed exactly as a single
// sweep would compute it (same FP32 operations in the same order), so K fused sweeps
// give bit-identical results to K separate launches.
//
// Decomposition ("2.5-D" blocking): a CTA owns a tile of (32 - 2K) x (48 - 2K) cells in
// x-y and a chunk of ZC planes in z. It walks z; at iteration z_in, stage 0 takes the
// region's plane z_in, and stage s (1..K) computes sweep s on plane z_in - s from stage
// s-1's planes z_in - s - 1 .. z_in - s + 1. Each stage keeps its last planes in
// registers (the z neighbours), exchanges x neighbours by warp shuffle and y neighbours
// through one shared-memory plane per stage. The 32 x 48 region carries a K-cell halo
// on every side in x-y (values there go stale one cell per stage and are never stored)
// and a K-plane halo in z. The input plane and the divergence plane of the next
// iteration are loaded one iteration ahead; each divergence plane is kept in a shared
// ring of K + 1 plane slots for the K stages that use it (slot z mod (K + 1): the slot a
// new plane overwrites was last read two iterations earlier, before two barriers).
//
// Threads: 768 = 24 warps x 32 lanes; lane l owns region column l and warp w region
// rows 2w, 2w+1 (2 cells per thread per plane).
//
// Boundaries, as in the reference: neighbours are clamped into the grid (walls and floor
// are Neumann), the top row of every sweep's output is 0 (the ambient boundary), and the
// z ends replicate the end plane (clamp). Cells of the region outside the grid compute
// garbage that no in-grid cell reads.
#pragma once

#include "fx_step_math.cuh"
#include "fx_storage.cuh"

#define FX_TB_THREADS 768
#define FX_TB_RX 32
#define FX_TB_RY 48

template <int K>
struct FxTbShape {
    static constexpr int TX = FX_TB_RX - 2 * K;
    static constexpr int TY = FX_TB_RY - 2 * K;
};

// Bricks of the COL shape for a grid: tiles in x, y and z chunks of zc planes.
__host__ __device__ inline int fx_tb_bricks(int X, int Y, int Z, int K, int zc) {
    const int tx = FX_TB_RX - 2 * K, ty = FX_TB_RY - 2 * K;
    return ((X + tx - 1) / tx) * ((Y + ty - 1) / ty) * ((Z + zc - 1) / zc);
}

template <typename PT>
FXD void fx_tb_store(void* p, int i, float v);
template <>
FXD void fx_tb_store<float>(void* p, int i, float v) {
    reinterpret_cast<float*>(p)[i] = v;
}
template <>
FXD void fx_tb_store<__half>(void* p, int i, float v) {
    reinterpret_cast<__half*>(p)[i] = __float2half_rn(v);
}

// Dynamic shared memory of one CTA: K stage planes followed by K + 1 divergence slots.
__host__ __device__ constexpr int fx_tb_smem_bytes(int K) { return (2 * K + 1) * FX_TB_RY * FX_TB_RX * 4; }

// One block-column of K sweeps. pin -> pout (distinct buffers). zeroIn: the input is
// known to be zero (the first sweep of a cleared solve); ROUND: round every sweep's
// result to FP16 (the reference's f16 branch stores every sweep, pressureShaders.ts:116).
// sm: K stage planes; dsm: K + 1 divergence plane slots.
template <int K, typename PT, bool ROUND>
FXD void fx_tb_column(const FxSimDev& S, const void* __restrict__ pin, void* __restrict__ pout, bool zeroIn, int tx,
                      int ty, int z0, int z1, float (*sm)[FX_TB_RY][FX_TB_RX], float (*dsm)[FX_TB_RY][FX_TB_RX]) {
    constexpr int TX = FxTbShape<K>::TX, TY = FxTbShape<K>::TY;
    const int X = S.X, Y = S.Y, Z = S.Z;
    const int sXY = X * Y;  // grids hold fewer than 2^31 cells: 32-bit offsets are exact
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ly0 = 2 * w;
    const int gx = tx * TX - K + lane, gy0 = ty * TY - K + ly0;
    const int cx = gx < 0 ? 0 : (gx > X - 1 ? X - 1 : gx);
    const bool selfL = gx <= 0;      // left neighbour clamps onto the cell itself
    const bool selfR = gx >= X - 1;  // right neighbour clamps onto the cell itself
    int off[2];                      // in-plane offset of each cell (clamped into the grid)
    bool selfB[2], top[2], keep[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int gy = gy0 + j, cy = gy < 0 ? 0 : (gy > Y - 1 ? Y - 1 : gy);
        off[j] = cy * X + cx;
        selfB[j] = gy <= 0;    // bottom neighbour clamps onto the cell itself
        top[j] = gy >= Y - 1;  // ambient top row: every sweep writes 0
        const int ly = ly0 + j;
        keep[j] = lane >= K && lane < FX_TB_RX - K && ly >= K && ly < FX_TB_RY - K && gx <= X - 1 && gy <= Y - 1;
    }
    const FxJacobiConst c{S.jc[0], S.jc[1], S.jc[2], S.jc[3]};
    const float rcpD = S.jcRcp;
    const bool fastDiv = S.jcFastDiv != 0;
    const int rowDn = ly0 > 0 ? ly0 - 1 : 0;                          // region row below row 0
    const int rowUp = ly0 + 2 < FX_TB_RY ? ly0 + 2 : FX_TB_RY - 1;    // region row above row 1
    const float* __restrict__ div = S.div;

    auto zclamp = [&](int z) { return z < 0 ? 0 : (z > Z - 1 ? Z - 1 : z); };

    // win[s][p][j]: stage s planes (p = 0: newest - 2, 1: newest - 1, 2: newest).
    float win[K][3][2];
#pragma unroll
    for (int s = 0; s < K; ++s)
#pragma unroll
        for (int j = 0; j < 2; ++j) win[s][0][j] = win[s][1][j] = win[s][2][j] = 0.0f;
    auto slot = [](int z) { return ((z % (K + 1)) + (K + 1)) % (K + 1); };
    float pnext[2], dnext[2];
    {
        const int pz = zclamp(z0 - K) * sXY, dz = zclamp(z0 - K - 1) * sXY;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            pnext[j] = zeroIn ? 0.0f : PStore<PT>::ld(pin, pz + off[j]);
            dnext[j] = __ldg(div + dz + off[j]);
        }
    }

    for (int zin = z0 - K; zin < z1 + K; ++zin) {
        float pcur[2];
        {
            const int sl = slot(zin - 1);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                pcur[j] = pnext[j];
                dsm[sl][ly0 + j][lane] = dnext[j];  // divergence of plane zin - 1
            }
        }
        if (zin + 1 < z1 + K) {  // prefetch the next iteration's input and divergence planes
            const int pz = zclamp(zin + 1) * sXY, dz = zclamp(zin) * sXY;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                pnext[j] = zeroIn ? 0.0f : PStore<PT>::ld(pin, pz + off[j]);
                dnext[j] = __ldg(div + dz + off[j]);
            }
        }
        // ---- stage 0: plane clamp(zin) of the input
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            win[0][0][j] = win[0][1][j];
            win[0][1][j] = win[0][2][j];
            win[0][2][j] = pcur[j];
            sm[0][ly0 + j][lane] = win[0][1][j];
        }
        __syncthreads();
        // ---- stages 1..K
#pragma unroll
        for (int s = 1; s <= K; ++s) {
            const int zs = zin - s;
            const int lo = z0 - K + s > 0 ? z0 - K + s : 0;
            const int hi = z1 + K - s;
            float v[2];
            if (zs >= lo && zs < hi && zs <= Z - 1) {
                const float below = sm[s - 1][rowDn][lane];
                const float above = sm[s - 1][rowUp][lane];
                const int sl = slot(zs);
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const float cen = win[s - 1][1][j];
                    const float fromLeft = __shfl_up_sync(0xffffffffu, cen, 1);
                    const float fromRight = __shfl_down_sync(0xffffffffu, cen, 1);
                    const float l = selfL ? cen : fromLeft;
                    const float r = selfR ? cen : fromRight;
                    const float b = selfB[j] ? cen : (j == 0 ? below : win[s - 1][1][0]);
                    const float t = j == 1 ? above : win[s - 1][1][1];
                    const float nb = fx_jacobi_numerator(c, l, r, b, t, win[s - 1][0][j], win[s - 1][2][j], dsm[sl][ly0 + j][lane]);
                    float u = top[j] ? 0.0f : (fastDiv ? fx_div_by_const(nb, c.denom, rcpD) : __fdiv_rn(nb, c.denom));
                    if (ROUND) u = PStore<__half>::round(u);
                    v[j] = u;
                }
                if (s == K && zs >= z0 && zs < z1) {
                    const int pl = zs * sXY;
#pragma unroll
                    for (int j = 0; j < 2; ++j)
                        if (keep[j]) fx_tb_store<PT>(pout, pl + off[j], v[j]);
                }
            } else {
                // outside this stage's needed planes: beyond the top end the end plane
                // repeats (clamp); below the chunk the values are never read
#pragma unroll
                for (int j = 0; j < 2; ++j) v[j] = s < K ? win[s][2][j] : 0.0f;
            }
            if (s < K) {
                if (zs == 0) {  // the grid's first plane: plane -1 clamps onto it
#pragma unroll
                    for (int j = 0; j < 2; ++j) win[s][1][j] = win[s][2][j] = v[j];
                }
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    win[s][0][j] = win[s][1][j];
                    win[s][1][j] = win[s][2][j];
                    win[s][2][j] = v[j];
                    sm[s][ly0 + j][lane] = win[s][1][j];
                }
                __syncthreads();
            }
        }
    }
}
