// fx_kernels_f32.cu — the plain FP32 Fire-X passes for sm_100a.
//
// Storage follows the reference bind groups (shaders.ts:16-24): flow and species are
// float4 per cell (AoS, 16 B, one 128-bit load per cell or trilinear tap), pressure,
// divergence and reaction are float per cell, liquid is uint32 per cell; cell index
// x + X*(y + Y*z). Compiled with --fmad=false so each reference expression is the same
// sequence of IEEE operations as in the WGSL source.
#include <cuda_runtime.h>

#include "fx_internal.h"
#include "fx_step_math.cuh"

namespace {

struct F32Acc {
    const float4* __restrict__ flowIn;
    const float4* __restrict__ speciesIn;
    const uint32_t* __restrict__ liq;
    FXD float4 flow(long long i) const { return __ldg(flowIn + i); }
    FXD float4 species(long long i) const { return __ldg(speciesIn + i); }
    FXD uint32_t liquid(long long i) const { return __ldg(liq + i); }
};

// simulate (shaders.ts:151-342). One thread per cell; 32x4x2 blocks keep the x rows of a
// warp contiguous (coalesced 16-byte loads) and the 6-neighbour / trilinear taps in L1.
__global__ void __launch_bounds__(256) fxk_simulate_f32(const FxParams* __restrict__ prm, FxGrid g,
                                                        const float4* __restrict__ flowIn,
                                                        const float4* __restrict__ speciesIn,
                                                        const uint32_t* __restrict__ liquid, float4* __restrict__ flowOut,
                                                        float4* __restrict__ speciesOut, float* __restrict__ reaction) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= g.X || y >= g.Y || z >= g.Z) return;
    F32Acc a{flowIn, speciesIn, liquid};
    FxCellOut o = fx_simulate_cell(*prm, g, x, y, z, a);
    long long id = (long long)x + (long long)g.X * ((long long)y + (long long)g.Y * z);
    flowOut[id] = o.flow;
    speciesOut[id] = o.species;
    reaction[id] = o.reaction;
}

// computeDivergence (shaders.ts:344-364): backward differences paired with the forward
// gradient of projectVelocity.
__global__ void __launch_bounds__(256) fxk_divergence_f32(const FxParams* __restrict__ prm, FxGrid g,
                                                          const float4* __restrict__ flow, float* __restrict__ div) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= g.X || y >= g.Y || z >= g.Z) return;
    float3 m = fx_metric(prm->u);
    long long id = g.idx(x, y, z);
    float4 c = __ldg(flow + id);
    float left = __ldg(&flow[g.idx(x - 1, y, z)].x);
    float bottom = __ldg(&flow[g.idx(x, y - 1, z)].y);
    float back = __ldg(&flow[g.idx(x, y, z - 1)].z);
    div[id] = (c.x - left) * m.x + (c.y - bottom) * m.y + (c.z - back) * m.z;
}

// One Jacobi sweep (solvePressureGlobal, shaders.ts:375-403). Each thread owns an (x, y)
// column over a chunk of z planes and slides p(z-1), p(z), p(z+1) through registers, so
// only the in-plane neighbours go through L1. Top row: ambient boundary, written 0.
__global__ void __launch_bounds__(256) fxk_jacobi_f32(const FxParams* __restrict__ prm, FxGrid g,
                                                      const float* __restrict__ pin, const float* __restrict__ div,
                                                      float* __restrict__ pout, int zchunk) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    int z0 = blockIdx.z * zchunk;
    if (x >= g.X || y >= g.Y || z0 >= g.Z) return;
    int z1 = min(g.Z, z0 + zchunk);
    const long long XY = (long long)g.X * g.Y;
    const long long col = (long long)x + (long long)g.X * y;
    if (y == g.Y - 1) {
        for (int z = z0; z < z1; ++z) pout[col + z * XY] = 0.0f;
        return;
    }
    FxJacobiConst c = fx_jacobi_const(prm->u);
    const int xl = x > 0 ? -1 : 0, xr = x < g.X - 1 ? 1 : 0;
    const long long yb = y > 0 ? -(long long)g.X : 0, yt = g.X;  // y + 1 <= Y - 1 here
    float pprev = __ldg(pin + col + (long long)max(z0 - 1, 0) * XY);
    float pcur = __ldg(pin + col + (long long)z0 * XY);
    for (int z = z0; z < z1; ++z) {
        long long id = col + z * XY;
        float pnext = __ldg(pin + col + (long long)min(z + 1, g.Z - 1) * XY);
        float l = __ldg(pin + id + xl), r = __ldg(pin + id + xr);
        float b = __ldg(pin + id + yb), t = __ldg(pin + id + yt);
        pout[id] = fx_jacobi_update(c, l, r, b, t, pprev, pnext, __ldg(div + id));
        pprev = pcur;
        pcur = pnext;
    }
}

// loadPressure (shaders.ts:366-373) for the projection: zero above the open top.
FXD float fx_loadp(const FxGrid& g, const float* __restrict__ p, int x, int y, int z) {
    return y >= g.Y ? 0.0f : __ldg(p + g.idx(x, y, z));
}

// projectVelocity (shaders.ts:461-501): u -= forward-difference grad p; the top row
// duplicates the projected row below (keeping its own T); wall-normal velocity zero.
__global__ void __launch_bounds__(256) fxk_project_f32(const FxParams* __restrict__ prm, FxGrid g,
                                                       const float4* __restrict__ flowIn, const float* __restrict__ p,
                                                       float4* __restrict__ flowOut) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    int z = blockIdx.z * blockDim.z + threadIdx.z;
    if (x >= g.X || y >= g.Y || z >= g.Z) return;
    float3 m = fx_metric(prm->u);
    long long id = g.idx(x, y, z);
    float4 f = __ldg(flowIn + id);
    int ys = (y == g.Y - 1) ? y - 1 : y;  // top row: gradient and velocity of the cell below
    float pc = fx_loadp(g, p, x, ys, z);
    float gx = (fx_loadp(g, p, x + 1, ys, z) - pc) * m.x;
    float gy = (fx_loadp(g, p, x, ys + 1, z) - pc) * m.y;
    float gz = (fx_loadp(g, p, x, ys, z + 1) - pc) * m.z;
    float4 src = (ys == y) ? f : __ldg(flowIn + g.idx(x, ys, z));
    float4 o = make_float4(src.x - gx, src.y - gy, src.z - gz, f.w);
    if (x == 0 || x == g.X - 1) o.x = 0.0f;
    if (z == 0 || z == g.Z - 1) o.z = 0.0f;
    if (y == 0) o.y = 0.0f;
    if (y == g.Y - 1) o.y = fx_max(0.0f, o.y);
    flowOut[id] = o;
}

// initializeFields (shaders.ts:135-149) plus the seeded velocity noise extension.
__global__ void fxk_init(FxGrid g, float4* __restrict__ flow, float4* __restrict__ species, uint64_t seed,
                         float noise, float tAmbient, float oxygen) {
    long long n = (long long)g.X * g.Y * g.Z;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < n; id += (long long)gridDim.x * blockDim.x) {
        float4 f = make_float4(0.0f, 0.0f, 0.0f, tAmbient);
        if (noise > 0.0f) {
            f.x = fx_velocity_noise(seed, (uint64_t)id, 0, noise);
            f.y = fx_velocity_noise(seed, (uint64_t)id, 1, noise);
            f.z = fx_velocity_noise(seed, (uint64_t)id, 2, noise);
        }
        flow[id] = f;
        species[id] = make_float4(0.0f, fx_max(oxygen, 0.0f), 0.0f, 0.0f);
    }
}

__global__ void fxk_emitter_mask(const FxParams* __restrict__ prm, FxGrid g, uint8_t* __restrict__ mask) {
    long long n = (long long)g.X * g.Y * g.Z;
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < n; id += (long long)gridDim.x * blockDim.x) {
        int x = (int)(id % g.X);
        int y = (int)((id / g.X) % g.Y);
        int z = (int)(id / ((long long)g.X * g.Y));
        uint8_t m = 0;
        if (prm->emitter_mode == FIREX_EMITTER_SPHERES)
            for (int s = 0; s < prm->num_spheres; ++s)
                if (fx_sphere_inside(prm->spheres[s], x, y, z)) m = 1;
        mask[id] = m;
    }
}

// Post-projection divergence norm over interior cells (the one-cell shell excluded,
// qualityShaders.ts:47-57): each block writes (sum of squares, max abs) in FP64 to
// partial[2*block]; fxk_norm_final sums the partials in a fixed order (deterministic).
__global__ void __launch_bounds__(256) fxk_norm_partial(const FxParams* __restrict__ prm, FxGrid g,
                                                        const float4* __restrict__ flow, double* __restrict__ partial) {
    float3 m = fx_metric(prm->u);
    const long long nInt = (long long)(g.X - 2) * (g.Y - 2) * (g.Z - 2);
    double ss = 0.0, mx = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nInt; k += (long long)gridDim.x * blockDim.x) {
        int x = 1 + (int)(k % (g.X - 2));
        int y = 1 + (int)((k / (g.X - 2)) % (g.Y - 2));
        int z = 1 + (int)(k / ((long long)(g.X - 2) * (g.Y - 2)));
        long long id = g.idx(x, y, z);
        float4 c = __ldg(flow + id);
        float d = (c.x - __ldg(&flow[id - 1].x)) * m.x + (c.y - __ldg(&flow[id - g.X].y)) * m.y +
                  (c.z - __ldg(&flow[id - (long long)g.X * g.Y].z)) * m.z;
        double dd = (double)d;
        ss += dd * dd;
        mx = fmax(mx, fabs(dd));
    }
    __shared__ double s_ss[256], s_mx[256];
    int t = threadIdx.x;
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

__global__ void fxk_norm_final(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
    __shared__ double s_ss[256], s_mx[256];
    int t = threadIdx.x;
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

// ---- launch wrappers --------------------------------------------------------------------
static inline dim3 cell_grid(const FxGrid& g, dim3 b) {
    return dim3((g.X + b.x - 1) / b.x, (g.Y + b.y - 1) / b.y, (g.Z + b.z - 1) / b.z);
}

void fx_launch_simulate_f32(cudaStream_t s, const FxParams* prm, FxGrid g, const float4* flowIn, const float4* speciesIn,
                            const uint32_t* liquid, float4* flowOut, float4* speciesOut, float* reaction) {
    dim3 b(32, 4, 2);
    fxk_simulate_f32<<<cell_grid(g, b), b, 0, s>>>(prm, g, flowIn, speciesIn, liquid, flowOut, speciesOut, reaction);
}

void fx_launch_divergence_f32(cudaStream_t s, const FxParams* prm, FxGrid g, const float4* flow, float* div) {
    dim3 b(32, 4, 2);
    fxk_divergence_f32<<<cell_grid(g, b), b, 0, s>>>(prm, g, flow, div);
}

void fx_launch_jacobi_f32(cudaStream_t s, const FxParams* prm, FxGrid g, const float* pin, const float* div, float* pout) {
    dim3 b(32, 8, 1);
    int zchunk = 8;
    dim3 grid((g.X + 31) / 32, (g.Y + 7) / 8, (g.Z + zchunk - 1) / zchunk);
    fxk_jacobi_f32<<<grid, b, 0, s>>>(prm, g, pin, div, pout, zchunk);
}

void fx_launch_project_f32(cudaStream_t s, const FxParams* prm, FxGrid g, const float4* flowIn, const float* p,
                           float4* flowOut) {
    dim3 b(32, 4, 2);
    fxk_project_f32<<<cell_grid(g, b), b, 0, s>>>(prm, g, flowIn, p, flowOut);
}

void fx_launch_init(cudaStream_t s, FxGrid g, float4* flow, float4* species, uint64_t seed, float noise, float tAmbient,
                    float oxygen) {
    fxk_init<<<148 * 8, 256, 0, s>>>(g, flow, species, seed, noise, tAmbient, oxygen);
}

void fx_launch_emitter_mask(cudaStream_t s, const FxParams* prm, FxGrid g, uint8_t* mask) {
    fxk_emitter_mask<<<148 * 8, 256, 0, s>>>(prm, g, mask);
}

int fx_norm_partial_blocks(FxGrid g) {
    long long nInt = (long long)(g.X - 2) * (g.Y - 2) * (g.Z - 2);
    long long b = (nInt + 255) / 256;
    return (int)(b < 148 * 8 ? (b < 1 ? 1 : b) : 148 * 8);
}

void fx_launch_divergence_norm(cudaStream_t s, const FxParams* prm, FxGrid g, const float4* flow, double* partial,
                               double* out) {
    int nb = fx_norm_partial_blocks(g);
    fxk_norm_partial<<<nb, 256, 0, s>>>(prm, g, flow, partial);
    fxk_norm_final<<<1, 256, 0, s>>>(partial, nb, out);
}

// Per-step parameter upload: the block travels as a kernel argument, so the host never
// has to keep a staging buffer alive and the launch can live inside a CUDA graph.
__global__ void fxk_upload_params(FxParams p, FxParams* __restrict__ dst) {
    const int* src = reinterpret_cast<const int*>(&p);
    int* d = reinterpret_cast<int*>(dst);
    for (int i = threadIdx.x; i < (int)(sizeof(FxParams) / 4); i += blockDim.x) d[i] = src[i];
}

void fx_launch_upload_params(cudaStream_t s, const FxParams& host, FxParams* dev) {
    fxk_upload_params<<<1, 128, 0, s>>>(host, dev);
}
