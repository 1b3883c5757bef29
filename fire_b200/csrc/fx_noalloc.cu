// fx_noalloc.cu — firex_divergence_norm_noalloc: the divergence norm of a caller-owned
// flow field, computed without any device allocation.
//
// Who needs it: a host that keeps its fields in memory it manages itself (its own pool,
// a framework's caching allocator holding the whole device, a fixed budget admitted up
// front) or that runs a frame or serving loop which must not stall. cudaMalloc and
// cudaFree can synchronise the device and can fail once the pool owns the memory, so
// such callers cannot let the library allocate per call, nor create a simulation handle
// just to get a norm. This entry point takes their device pointer and uses a small
// scratch array that lives in the library's own device image instead.
//
// Scratch: one file-scope __device__ array, present on every GPU that loads the library
// until the process exits. It holds one (sum of squares, max abs) pair per interior z
// plane, FX_NOALLOC_MAX_PLANES planes at most, plus the final pair: 32 KiB. Every call
// writes the pairs of its own planes before it reads them, so nothing has to start at
// zero. All calls share the array: calls whose kernels overlap on a GPU (other streams,
// other host threads) race on it, so callers serialise them.
//
// Host code must not pass the array's name to a kernel: on the host it is a stand-in,
// not a device address. Its device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, on the first call that runs there;
// that first call should come before any stream capture on the caller's side.
#include <cuda.h>  // CUdeviceptr / CUresult, for the driver's address-range query
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/firex.h"
#include "fx_internal.h"

#define FX_NOALLOC_MAX_PLANES FIREX_NOALLOC_MAX_PLANES
#define FX_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double fx_noalloc_scratch[2 * FX_NOALLOC_MAX_PLANES + 2];

namespace {

// One CTA per interior plane z = 1 .. Z-2: the plane's interior cells, the backward
// divergence of qualityShaders.ts:47-57 / shaders.ts:344-364 as FP32, squares and
// maxima accumulated in FP64, then a fixed-order tree inside the CTA (deterministic).
__global__ void __launch_bounds__(256) fxk_noalloc_plane(const float4* __restrict__ flow, int X, int Y, float mx,
                                                         float my, float mz, double* __restrict__ scratch) {
    const int z = 1 + blockIdx.x;
    const long long XY = (long long)X * Y;
    const long long nPlane = (long long)(X - 2) * (Y - 2);
    double ss = 0.0, mxa = 0.0;
    for (long long k = threadIdx.x; k < nPlane; k += blockDim.x) {
        const int x = 1 + (int)(k % (X - 2));
        const int y = 1 + (int)(k / (X - 2));
        const long long id = x + (long long)X * y + XY * z;
        const float4 c = flow[id];
        const float d = (c.x - flow[id - 1].x) * mx + (c.y - flow[id - X].y) * my + (c.z - flow[id - XY].z) * mz;
        const double dd = (double)d;
        ss += dd * dd;
        mxa = fmax(mxa, fabs(dd));
    }
    __shared__ double s_ss[256], s_mx[256];
    const int t = threadIdx.x;
    s_ss[t] = ss;
    s_mx[t] = mxa;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w) {
            s_ss[t] += s_ss[t + w];
            s_mx[t] = fmax(s_mx[t], s_mx[t + w]);
        }
        __syncthreads();
    }
    if (t == 0) {
        scratch[2 * blockIdx.x] = s_ss[0];
        scratch[2 * blockIdx.x + 1] = s_mx[0];
    }
}

// Reduces the nPlanes pairs in a fixed order into the last pair of the scratch array.
__global__ void __launch_bounds__(256) fxk_noalloc_final(double* __restrict__ scratch, int nPlanes) {
    __shared__ double s_ss[256], s_mx[256];
    const int t = threadIdx.x;
    double ss = 0.0, mxa = 0.0;
    for (int b = t; b < nPlanes; b += 256) {
        ss += scratch[2 * b];
        mxa = fmax(mxa, scratch[2 * b + 1]);
    }
    s_ss[t] = ss;
    s_mx[t] = mxa;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w) {
            s_ss[t] += s_ss[t + w];
            s_mx[t] = fmax(s_mx[t], s_mx[t + w]);
        }
        __syncthreads();
    }
    if (t == 0) {
        scratch[2 * FX_NOALLOC_MAX_PLANES] = sqrt(s_ss[0]);
        scratch[2 * FX_NOALLOC_MAX_PLANES + 1] = s_mx[0];
    }
}

std::mutex g_setup_mu;
double* g_scratch[FX_NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array on `device`, looked up once with that device
// current (the caller has made it current).
cudaError_t scratch_on(int device, double** out) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, fx_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch[device] = static_cast<double*>(p);
    }
    *out = g_scratch[device];
    return cudaSuccess;
}

int fail(int code, const std::string& msg) {
    fx_set_thread_error("firex_divergence_norm_noalloc: " + msg);
    return code;
}

// cuMemGetAddressRange through the runtime's driver entry point (no link-time dependency
// on the driver library): the base and size of the allocation that holds a device address.
using AddressRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
AddressRangeFn address_range_fn() {
    static AddressRangeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<AddressRangeFn>(p);
        cudaGetLastError();
    });
    return fn;
}

}  // namespace

extern "C" int firex_divergence_norm_noalloc(const void* flow, const int32_t dims[3], const float metric[3],
                                             void* stream, double out[3]) {
    if (!flow || !dims || !metric || !out) return fail(FIREX_ERR_BAD_ARG, "flow, dims, metric and out are required");
    const int X = dims[0], Y = dims[1], Z = dims[2];
    if (X < 1 || Y < 1 || Z < 1) return fail(FIREX_ERR_BAD_ARG, "grid axes must be positive");
    if (reinterpret_cast<uintptr_t>(flow) % 16 != 0) return fail(FIREX_ERR_BAD_ARG, "flow must be 16-byte aligned");
    if (Z - 2 > FX_NOALLOC_MAX_PLANES)
        return fail(FIREX_ERR_BAD_ARG, "Z = " + std::to_string(Z) + " has " + std::to_string(Z - 2) +
                                           " interior planes; the static scratch holds at most " +
                                           std::to_string(FX_NOALLOC_MAX_PLANES));
    out[0] = out[1] = 0.0;
    out[2] = (X > 2 && Y > 2 && Z > 2) ? (double)(X - 2) * (double)(Y - 2) * (double)(Z - 2) : 0.0;
    if (out[2] == 0.0) return FIREX_OK;  // no interior cells: nothing to launch

    // The kernels run on the device that owns `flow`.
    cudaPointerAttributes attr{};
    cudaError_t e = cudaPointerGetAttributes(&attr, flow);
    if (e != cudaSuccess || (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) ||
        attr.devicePointer == nullptr || attr.device < 0) {
        cudaGetLastError();
        return fail(FIREX_ERR_BAD_ARG, "flow is not device memory");
    }
    if (attr.device >= FX_NOALLOC_MAX_DEVICES) return fail(FIREX_ERR_UNSUPPORTED, "device ordinal above 63");
    // The allocation that holds flow must hold every record the dims ask for: the kernels
    // would otherwise read past its end.
    const unsigned long long need = (unsigned long long)X * Y * Z * 16ull;
    if (AddressRangeFn range = address_range_fn()) {
        CUdeviceptr base = 0;
        size_t size = 0;
        const CUdeviceptr dp = (CUdeviceptr)(uintptr_t)attr.devicePointer;
        if (range(&base, &size, dp) != CUDA_SUCCESS)
            return fail(FIREX_ERR_BAD_ARG, "flow is not inside a device allocation");
        if (dp - base > size || need > (unsigned long long)(size - (dp - base)))
            return fail(FIREX_ERR_BAD_ARG, "dims need " + std::to_string(need) + " bytes of flow records; the allocation "
                                           "holds " + std::to_string((unsigned long long)(size - (dp - base))) +
                                           " from flow to its end");
    }
    int prev = -1;
    e = cudaGetDevice(&prev);
    if (e == cudaSuccess && prev != attr.device) e = cudaSetDevice(attr.device);
    double* scratch = nullptr;
    if (e == cudaSuccess) e = scratch_on(attr.device, &scratch);
    if (e == cudaSuccess) {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const int nPlanes = Z - 2;
        cudaGetLastError();  // an earlier error of the caller's own work is not this call's
        fxk_noalloc_plane<<<nPlanes, 256, 0, st>>>(static_cast<const float4*>(attr.devicePointer), X, Y, metric[0],
                                                   metric[1], metric[2], scratch);
        fxk_noalloc_final<<<1, 256, 0, st>>>(scratch, nPlanes);
        e = cudaGetLastError();
        double res[2] = {0.0, 0.0};
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(res, scratch + 2 * FX_NOALLOC_MAX_PLANES, sizeof(res), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) {
            out[0] = res[0];
            out[1] = res[1];
        }
    }
    if (prev >= 0 && prev != attr.device) cudaSetDevice(prev);
    if (e != cudaSuccess) return fail(FIREX_ERR_CUDA, cudaGetErrorString(e));
    return FIREX_OK;
}
